// tracing.cuh -- device pieces of the delta-tracking tracer shared by the
// render kernels (tracer_kernels.cu) and the interactive frame
// (interactive.cu): free flight with null collisions, one path sample.
#pragma once
#include "common.cuh"

namespace mrp {

// Free-flight lookups stay plain: delta tracking takes few steps in empty
// bricks, so the brick test cost more than it saved (measured).
// DT: the density grid's storage type, or void (read from the volume per fetch).
template <class DT = void>
MRP_D float density_t(const VolumeDev& v, f3 p) { return density_as<DT>(v, p); }

// DeterminateNextVertex.  SampleHenyeyGreenstein(Rand, Rand, ...) takes the
// first draw as e1 and the second as e0 (x86-64 g++ argument order).
MRP_D bool next_vertex(const VolumeDev& v, Stream& st, float alpha, float g, f3 pos, f3 dir, float dis, f3* npos,
                       f3* ndir, Tally* tl) {
    float smax = fm(v.max_density, alpha);
    float t = 0.0f;
    int loop = 0;
    while (loop++ < 10000) {
        float rk = st.next();
        t = fs(t, fd(logf(fs(1.0f, rk)), smax));
        if (t > dis) { *npos = mk3(0, 0, 0); *ndir = mk3(0, 0, 0); return false; }
        rk = st.next();
        float d = density_t(v, add(pos, mul(dir, t)));
        if (tl) tl->fetches++;
        float S = fm(d, alpha);
        if (fd(S, smax) > rk) break;
        if (d < 0) t = fs(t, d);
    }
    float e1 = st.next();
    float e0 = st.next();
    *ndir = sample_hg(e0, e1, dir, g);
    *npos = add(mul(dir, t), pos);
    return true;
}

MRP_D f3 camera_ray_t(const ViewDev& w, int row, int col) { return camera_ray_dir(w, row, col); }

// Radiance of sample k of one pixel (CalculateRadiance's loop body).
MRP_D f3 trace_sample(const VolumeDev& v, const ViewDev& w, int pix, int k, f3 ori, f3 dir, float dis, f3 L, Tally* tl) {
    Stream st(kPixelStream, (uint32_t)pix, (uint32_t)k, (uint32_t)w.frame, w.seed);
    Stream nst(kNeeStream, (uint32_t)pix, (uint32_t)k, (uint32_t)w.frame, w.seed);   // nee_mode 1 only
    f3 res = mk3(0, 0, 0);
    f3 p = add(ori, mul(dir, dis)), rd = dir, csr = mk3(1, 1, 1);
    for (int b = 0; b < w.multi_scatter; ++b) {
        f3 np, nd;
        float md = ray_box_distance(p, rd);
        if (tl) tl->steps++;
        if (!next_vertex(v, st, w.alpha, w.g, p, rd, md, &np, &nd, tl)) {
            res = add(res, mul(sky_radiance(v, rd), csr));
            break;
        }
        p = np;
        csr = mul(csr, v.scatter_rate);
        float ph = hg(dot(rd, L), w.g);
        float tr = v.nee_mode ? transmittance(v, nst, p, L, ray_box_distance(p, L), w.alpha)
                              : tex3<true>(v.baked, v.baked_res, p);
        if (tl) tl->lookups++;
        res = add(res, mul(mul(w.light_color, csr), fm(tr, ph)));
        rd = nd;
    }
    return res;
}

}  // namespace mrp
