// The end-of-step sponge (state relaxation) of a flat C-grid level, sm_100a:
// apply_rayleigh_damping then apply_lateral_damping
// (src/core/infra/rayleigh_damping.cpp:720-1119, 1194-1476), the pass
// dynamics.cpp:7323-7340 runs after the EOS projection.  The reference runs
// three passes over the grid (upper sponge, w-only lid absorber, lateral
// band); each touches a cell's own u, v, w, theta only, so one thread per cell
// applies the three in that order.  The relaxation factors depend on the
// level (or the distance from the nearest lateral face) only and are formed
// on the host with the C library's expm1, the function the reference calls;
// a cell adds factor * (ref - old) in FP64, rounded to FP32 and added in
// FP32, as the reference's Field3D proxy adds it.  One pass reads and writes
// 16 bytes per cell: HBM-bound.
#pragma once

#include "stencil_common.cuh"

namespace nimbus
{

// Per-level tables on the device: factor of the upper sponge at scalar and at
// w levels, w-only factor, references, then the lateral factors by distance.
struct RelaxTables
{
    const double* upper;    // [nz]
    const double* upper_w;  // [nz]
    const double* w_only;   // [nz]
    const double* u_ref;    // [nz]
    const double* v_ref;    // [nz]
    const double* th_ref;   // [nz]
    const double* lateral;  // [lateral_width]
    const unsigned char* upper_on;   // [nz] level inside the upper sponge
    const unsigned char* w_only_on;  // [nz] level inside the lid absorber
    int lateral_width;
    int do_upper, do_w_only, do_lateral;
};

__device__ __forceinline__ void relax_add(float& x, double delta) { x = __fadd_rn(x, (float)delta); }

static __global__ void __launch_bounds__(256) state_relaxation_kernel(Dims d, RelaxTables R, float* __restrict__ u,
                                                                      float* __restrict__ v, float* __restrict__ w,
                                                                      float* __restrict__ theta)
{
    const int n = d.cells();
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    {
        int i, j, k;
        decompose(d, c, i, j, k);
        const int di = min(i, d.nx - 1 - i), dj = min(j, d.ny - 1 - j);
        const int dist = min(di, dj);
        const bool upper = R.do_upper && R.upper_on[k];
        const bool lid = R.do_w_only && R.w_only_on[k];
        const bool lateral = R.do_lateral && dist < R.lateral_width;
        if (!upper && !lid && !lateral) continue;
        float uu = u[c], vv = v[c], ww = w[c], th = theta[c];
        const double ur = R.u_ref[k], vr = R.v_ref[k], tr = R.th_ref[k];
        if (upper)
        {
            const double f = R.upper[k], fw = R.upper_w[k];
            const double u0 = uu, v0 = vv, w0 = ww, t0 = th;
            relax_add(uu, f * (ur - u0));
            relax_add(vv, f * (vr - v0));
            relax_add(ww, fw * (0.0 - w0));
            relax_add(th, f * (tr - t0));
        }
        if (lid)
        {
            const double w0 = ww;
            relax_add(ww, R.w_only[k] * (0.0 - w0));
        }
        if (lateral)
        {
            const double f = R.lateral[dist];
            const double u0 = uu, v0 = vv, w0 = ww, t0 = th;
            relax_add(uu, f * (ur - u0));
            relax_add(vv, f * (vr - v0));
            relax_add(ww, f * (0.0 - w0));
            relax_add(th, f * (tr - t0));
        }
        u[c] = uu;
        v[c] = vv;
        w[c] = ww;
        theta[c] = th;
    }
}

}  // namespace nimbus
