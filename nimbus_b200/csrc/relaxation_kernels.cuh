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

#include <algorithm>
#include <cmath>
#include <vector>

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

// The three passes on one cell (i, j, k) of an nx x ny level, in the
// reference's order.  Returns false (values untouched) where no pass applies.
__device__ __forceinline__ bool relax_cell(const RelaxTables& R, int nx, int ny, int i, int j, int k, float& uu,
                                           float& vv, float& ww, float& th)
{
    const int dist = min(min(i, nx - 1 - i), min(j, ny - 1 - j));
    const bool upper = R.do_upper && R.upper_on[k];
    const bool lid = R.do_w_only && R.w_only_on[k];
    const bool lateral = R.do_lateral && dist < R.lateral_width;
    if (!upper && !lid && !lateral) return false;
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
    return true;
}

static __global__ void __launch_bounds__(256) state_relaxation_kernel(Dims d, RelaxTables R, float* __restrict__ u,
                                                                      float* __restrict__ v, float* __restrict__ w,
                                                                      float* __restrict__ theta)
{
    const int n = d.cells();
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    {
        int i, j, k;
        decompose(d, c, i, j, k);
        float uu = u[c], vv = v[c], ww = w[c], th = theta[c];
        if (!relax_cell(R, d.nx, d.ny, i, j, k, uu, vv, ww, th)) continue;
        u[c] = uu;
        v[c] = vv;
        w[c] = ww;
        theta[c] = th;
    }
}

}  // namespace nimbus

namespace nimbus_host
{

// damping_relaxation_factor (rayleigh_damping.cpp:145-163): false where the
// reference throws.
inline bool relaxation_factor(double alpha, double dt, int implicit_mode, double* out)
{
    if (!std::isfinite(alpha) || alpha < 0.0 || !std::isfinite(dt) || dt <= 0.0) return false;
    const double scaled = alpha * dt;
    if (!std::isfinite(scaled)) return false;
    *out = implicit_mode ? scaled / (1.0 + scaled) : -std::expm1(-scaled);
    return true;
}

// Host image of one level's sponge tables: doubles [upper nz | upper_w nz |
// w_only nz | u_ref nz | v_ref nz | theta_ref nz | lateral W (at least 1)]
// then the level flags [upper_on nz | w_only_on nz] as bytes.  The factors the
// reference forms cell by cell depend on the level (or lateral distance)
// only; they are formed here once with the same expm1 and checked where the
// reference would evaluate them.  Returns an error message or null.
struct RelaxImage
{
    std::vector<double> tab;
    std::vector<unsigned char> on;
    int width = 0;
    bool upper = false, lid = false, lateral = false;
    size_t bytes() const { return tab.size() * sizeof(double) + on.size(); }
};

inline const char* build_relax_image(int nx, int ny, int nz, const double* alpha, const double* upper_w_alpha,
                                     const double* w_only_alpha, const double* u_ref, const double* v_ref,
                                     const double* theta_ref, int lateral_width, const double* lateral_alpha,
                                     int do_upper, int do_w_only, int do_lateral, int staggered, int implicit_mode,
                                     double dt, RelaxImage& out)
{
    if (lateral_width < 0) return "lateral sponge width must be >= 0";
    out.upper = do_upper != 0;
    out.lid = do_w_only != 0;
    out.lateral = do_lateral != 0 && lateral_width > 0;
    if ((out.upper && (!alpha || !upper_w_alpha)) || (out.lid && !w_only_alpha) ||
        (out.lateral && !lateral_alpha) || ((out.upper || out.lateral) && (!u_ref || !v_ref || !theta_ref)))
        return "a profile of an enabled sponge pass is null";
    out.width = out.lateral ? lateral_width : 0;
    out.tab.assign(6 * static_cast<size_t>(nz) + static_cast<size_t>(out.width > 0 ? out.width : 1), 0.0);
    out.on.assign(2 * static_cast<size_t>(nz), 0);
    double* up = out.tab.data();
    double* up_w = up + nz;
    double* lid_f = up_w + nz;
    double* refs = lid_f + nz;
    double* lat = refs + 3 * nz;
    for (int k = 0; k < nz; ++k)
    {
        if (out.upper && !(alpha[k] <= 0.0 && upper_w_alpha[k] <= 0.0))
        {
            out.on[k] = 1;
            if (!relaxation_factor(alpha[k], dt, implicit_mode, &up[k]))
                return "upper sponge: alpha and dt must be finite, alpha >= 0, dt > 0";
            if (!staggered) up_w[k] = up[k];
            else if (!relaxation_factor(upper_w_alpha[k], dt, implicit_mode, &up_w[k]))
                return "upper sponge: alpha and dt must be finite, alpha >= 0, dt > 0";
        }
        if (out.lid && w_only_alpha[k] > 0.0)
        {
            out.on[nz + k] = 1;
            if (!relaxation_factor(w_only_alpha[k], dt, implicit_mode, &lid_f[k]))
                return "w-only sponge: alpha and dt must be finite, dt > 0";
        }
        if (out.upper || out.lateral)
        {
            refs[k] = u_ref[k];
            refs[nz + k] = v_ref[k];
            refs[2 * nz + k] = theta_ref[k];
        }
    }
    // Only the distances that occur on this grid are evaluated, as in the
    // reference (a band wider than half the domain never reaches its inner
    // entries).
    const int reach = std::min((nx - 1) / 2, (ny - 1) / 2);
    for (int dd = 0; dd < out.width && dd <= reach; ++dd)
        if (!relaxation_factor(lateral_alpha[dd], dt, implicit_mode, &lat[dd]))
            return "lateral sponge: alpha and dt must be finite, alpha >= 0, dt > 0";
    return nullptr;
}

// Device views of an image uploaded to `dev`.
inline nimbus::RelaxTables relax_tables(const RelaxImage& img, const unsigned char* dev, int nz)
{
    const size_t tab_bytes = img.tab.size() * sizeof(double);
    const double* t = reinterpret_cast<const double*>(dev);
    nimbus::RelaxTables R;
    R.upper = t;
    R.upper_w = t + nz;
    R.w_only = t + 2 * nz;
    R.u_ref = t + 3 * nz;
    R.v_ref = t + 4 * nz;
    R.th_ref = t + 5 * nz;
    R.lateral = t + 6 * nz;
    R.upper_on = dev + tab_bytes;
    R.w_only_on = dev + tab_bytes + nz;
    R.lateral_width = img.width;
    R.do_upper = img.upper;
    R.do_w_only = img.lid;
    R.do_lateral = img.lateral;
    return R;
}

}  // namespace nimbus_host
