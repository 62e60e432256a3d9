"""RadiancePredictInternal (core/radiancePredict.cu:301-422) as a batched
PyTorch network on the CPU: the CPU baseline of the predictor's network
("PyTorch-CPU batched port of the exact MLP"), timed beside the OpenMP
oracle and the GPU kernels.

TEST INFRASTRUCTURE ONLY (a CPU baseline and a checker): imported by tests/
and the CPU legs of bench.py, never by the product package.

The network is the oracle's (oracle/mrpnn_oracle.cpp mlp_one) in batched
form, weights from the model file: per SE block the slice [from, from + w) of
the three feature channels (X_Val, X_Val_Sub, X_Val_Hg), its (avg, max)
pools plus (g, gamma) through the gate MLP 8 -> 8 -> 3, per channel
relu(W (x * gate + prev) + b), then the raw slice added (ADD3) or
concatenated (REP3); the finals, then the tail per distinct albedo channel
(LGGS, the LSEFin gate over the 75 pools, LC0..LC2, LX, six residual pairs,
LX12).  Float32 throughout; sums run in PyTorch's order, so results agree
with the oracle's sequential sums to ~1e-6 relative, not bit for bit.
"""
import os
import struct

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
MODEL = os.path.join(os.path.dirname(HERE), "mrpnn_b200", "data", "mrpnn_model.bin")

# (from, width, pool index, widen, SE gate weights, branch weights per channel)
MAIN = [(0, 8, 0, False, "LSE0", "L01"), (8, 8, 3, True, "LSE1", "L11"), (16, 16, 6, False, "LSE2", "L21"),
        (32, 16, 9, False, "LSE3", "L31"), (48, 16, 12, True, "LSE4", "L41"), (64, 32, 15, False, "LSE5", "L51"),
        (96, 32, 18, False, "LSE6", "L61"), (128, 32, 21, False, "LSE7", "L71")]
DI = [(160, 8, 24, False, "LDSE0", "LD01"), (168, 8, 27, False, "LDSE1", "LD11"), (176, 8, 30, False, "LDSE2", "LD21"),
      (184, 8, 33, False, "LDSE3", "LD31")]


def _channel_names(base):
    """L01 -> (L01, L_Tr01, L_Hg01); LD01 -> (LD01, LD_Tr01, LD_Hg01)."""
    head = "LD" if base.startswith("LD") else "L"
    tail = base[len(head):]
    return base, f"{head}_Tr{tail}", f"{head}_Hg{tail}"


def load_model(path=MODEL):
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != b"MRPNNMD1":
        raise ValueError(f"{path}: not a model file")
    n = struct.unpack_from("<I", data, 8)[0]
    off, out = 12, {}
    for _ in range(n):
        ln = struct.unpack_from("<H", data, off)[0]
        off += 2
        name = data[off:off + ln].decode()
        off += ln
        cnt = struct.unpack_from("<I", data, off)[0]
        off += 4
        out[name] = torch.from_numpy(np.frombuffer(data, "<f4", cnt, off).copy())
        off += 4 * cnt
    return out


class RadiancePredictor:
    def __init__(self, path=MODEL):
        self.t = load_model(path)

    def _w(self, name, to, frm):
        return self.t[name].view(to, frm)

    def _block(self, X, pool, g, gamma, blk, prev):
        frm, w, pid, widen, se, base = blk
        sl = X[:, :, frm:frm + w]                              # [n, 3, w]
        avg = sl.sum(-1) / w
        mx = torch.maximum(sl.amax(-1), torch.tensor(-10000.0))
        pool[:, pid:pid + 3] = avg
        pool[:, 36 + pid:39 + pid] = mx
        p8 = torch.cat([avg, mx, g[:, None], gamma[:, None]], 1)
        h = torch.relu(p8 @ self._w(se + "1W", 8, 8).T)
        gate = torch.sigmoid(h @ self._w(se + "2W", 3, 8).T)  # [n, 3]
        nxt = []
        for c, name in enumerate(_channel_names(base)):
            x = sl[:, c] * gate[:, c:c + 1]
            if prev is not None:
                x = x + prev[c]
            o = torch.relu(x @ self._w(name + "W", w, w).T + self.t[name + "B"])
            nxt.append(torch.cat([o, sl[:, c]], 1) if widen else o + sl[:, c])
        return nxt

    @torch.no_grad()
    def __call__(self, feat, gamma, g, sr):
        """feat [n, 576] (X_Val, X_Val_Sub, X_Val_Hg), gamma [n] -> [n, 3]."""
        feat = torch.as_tensor(np.asarray(feat, np.float32))
        n = feat.shape[0]
        X = feat.view(n, 3, 192)
        gamma = torch.as_tensor(np.asarray(gamma, np.float32))
        gv = torch.full((n,), float(g), dtype=torch.float32)
        pool = torch.zeros((n, 75), dtype=torch.float32)
        pool[:, 72] = gv
        pool[:, 73] = gamma
        prev = None
        for blk in MAIN:
            prev = self._block(X, pool, gv, gamma, blk, prev)
        comb = [torch.relu(prev[c] @ self._w(nm + "W", 32, 32).T + self.t[nm + "B"])
                for c, nm in enumerate(("L81", "L_Tr81", "L_Hg81"))]
        prev = None
        for blk in DI:
            prev = self._block(X, pool, gv, gamma, blk, prev)
        comb += [torch.relu(prev[c] @ self._w(nm + "W", 8, 8).T + self.t[nm + "B"])
                 for c, nm in enumerate(("LD41", "LD_Tr41", "LD_Hg41"))]
        comb = torch.cat(comb, 1)                              # [n, 120]
        srv = [float(x) for x in sr]
        P = {}
        for s in srv:
            if s in P:
                continue
            s4 = float(np.float32(s) ** np.float32(4.0))
            pool[:, 74] = s4
            lg = torch.relu(pool[:, 72:75] @ self._w("LGGSW", 8, 3).T + self.t["LGGSB"])
            hf = torch.relu(pool @ self._w("LSEFin1W", 16, 75).T)
            gf = torch.sigmoid(hf @ self._w("LSEFin2W", 6, 16).T)
            scale = torch.cat([gf[:, k:k + 1].expand(n, ln) for k, ln in enumerate((32, 32, 32, 8, 8, 8))], 1)
            x = torch.cat([comb * scale, lg], 1)
            x = torch.relu(x @ self._w("LC0W", 128, 128).T + self.t["LC0B"])
            x = torch.relu(x @ self._w("LC1W", 64, 128).T + self.t["LC1B"])
            x = torch.relu(x @ self._w("LC2W", 32, 64).T + self.t["LC2B"])
            x = torch.relu(x @ self._w("LXW", 16, 32).T + self.t["LXB"])
            for k in range(6):
                y = torch.relu(x @ self._w(f"LX{2 * k}W", 16, 16).T + self.t[f"LX{2 * k}B"])
                z = torch.relu(y @ self._w(f"LX{2 * k + 1}W", 16, 16).T + self.t[f"LX{2 * k + 1}B"])
                x = x + z
            P[s] = torch.relu(x @ self._w("LX12W", 1, 16).T + self.t["LX12B"])[:, 0]
        out = torch.stack([torch.clamp(torch.exp(P[s]) - 1.0, min=0.0) * float(np.float32(s) ** np.float32(4.0))
                           for s in srv], 1)
        return out.numpy()
