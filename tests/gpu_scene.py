"""Shared set-up of the GPU parity tests: one synthetic fBm scene built on the
device through the C ABI and the same scene handed to the CPU oracle."""
import numpy as np

from oracle import oracle as O

LIGHT = np.array([0.3, 0.8, 0.5], np.float32)
LIGHT = (LIGHT / np.float32(np.sqrt(np.float32(np.dot(LIGHT, LIGHT))))).astype(np.float32)


def view_frame(fov_deg=45.0, pos=(0.75, 0.75, 0.75)):
    import mrpnn_b200 as M
    ori, up, right = M.camera_frame(pos)
    s = np.float32(np.tan(np.deg2rad(fov_deg) / 2))
    return ori, (up * s).astype(np.float32), (right * s).astype(np.float32)


class Scene:
    """GPU volume + oracle SceneBuf over the GPU's own resources (each
    resource is checked against the oracle separately)."""

    def __init__(self, R=64, seed=0, freq=4.0, alpha=64.0, g=0.857, sr=0.99, sky=0.05, bake_res=0):
        import mrpnn_b200 as M
        M.init()
        self.R, self.alpha, self.g = R, alpha, g
        self.vol = M.VolumeRender(R)
        self.vol.generate_fbm(seed, freq)
        self.vol.Update()
        self.vol.SetScatterRate(sr)
        self.vol.SetSky(sky)
        self.vol.UpdateHGLut(g)
        self.vol.Update_TR(LIGHT, alpha)
        self.density = self.vol.read(M.api.RES_DENSITY)
        self.mips = np.concatenate([self.vol.read(M.api.RES_MIP, m) for m in range(9)])
        self.tr = np.concatenate([self.vol.read(M.api.RES_TR, i) for i in range(8)])
        self.lut = self.vol.read(M.api.RES_LUT)
        baked, bres = None, 0
        if bake_res:
            self.vol.SetBakeResolution(bake_res)
            self.vol.Update_CachedTR(LIGHT, alpha)
            baked, bres = self.vol.read(M.api.RES_BAKED_TR), bake_res
        self.baked = baked
        self.max_density = self.vol.max_density
        self.orc = O.SceneBuf(self.density, R, self.max_density, self.mips, self.tr, self.lut, baked=baked,
                              baked_res=bres, scatter_rate=(sr, sr, sr), sky=(sky, sky, sky))
