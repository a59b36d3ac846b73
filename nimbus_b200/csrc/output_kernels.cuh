// Cell-centre velocities for output: the C-grid output staging of the
// reference's history and live export (interpolate_u/v/w_face_to_center,
// src/core/output/stagger_interpolation.cpp; called at
// src/core/runtime/headless_runtime.cpp:2577-2601 before every export).
//
// u: centre i is 0.5f * (face i-1 + face i), cell 0 keeps face 0 (the
// maintained west boundary face); v likewise in j; w: centre k > 0 is
// 0.5f * (face k-1 + face k) and centre 0 is 0.5 (ground + face 0) formed in
// FP64 and rounded once, ground being the column's lower-face velocity (0 on
// flat ground, the terrain-tangent velocity otherwise).
//
// HBM-bound (12 B read + 12 B written per cell for all three components; the
// i-1 plane and j-1 row come back from L2).  Each thread takes V consecutive
// cells of one column (V = 4, 2 or 1, the widest that divides nz), so every
// access is a V-wide vector load or store except the w[k-1] neighbour.
#pragma once

#include "stencil_common.cuh"

namespace nimbus
{

struct CentreFields
{
    const float* u;
    const float* v;
    const float* w;
    float* uc;             // null: component skipped
    float* vc;
    float* wc;
    const double* ground;  // [nx][ny] lower-face w; null: flat ground
};

template <int V>
__device__ __forceinline__ void load_run(const float* p, float (&x)[V])
{
    if constexpr (V == 4)
    {
        const float4 t = __ldg(reinterpret_cast<const float4*>(p));
        x[0] = t.x;
        x[1] = t.y;
        x[2] = t.z;
        x[3] = t.w;
    }
    else if constexpr (V == 2)
    {
        const float2 t = __ldg(reinterpret_cast<const float2*>(p));
        x[0] = t.x;
        x[1] = t.y;
    }
    else
    {
        x[0] = __ldg(p);
    }
}

template <int V>
__device__ __forceinline__ void store_run(float* p, const float (&x)[V])
{
    if constexpr (V == 4)
        *reinterpret_cast<float4*>(p) = make_float4(x[0], x[1], x[2], x[3]);
    else if constexpr (V == 2)
        *reinterpret_cast<float2*>(p) = make_float2(x[0], x[1]);
    else
        *p = x[0];
}

// 0.5f * (a + b) in FP32, the reference's face mean.
__device__ __forceinline__ float face_mean(float a, float b) { return __fmul_rn(0.5f, __fadd_rn(a, b)); }

template <int V>
__global__ void __launch_bounds__(256) cell_centre_kernel(Dims d, CentreFields F)
{
    const int runs = d.cells() / V;
    const int plane = d.sx();
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < runs; r += gridDim.x * blockDim.x)
    {
        const int c = r * V;
        int i, j, k;
        decompose(d, c, i, j, k);
        // Every load first, so the independent HBM requests are in flight together.
        float u[V], up[V], v[V], vp[V], w[V];
        float wp = 0.0f;
        double g = 0.0;
        if (F.uc)
        {
            load_run<V>(F.u + c, u);
            if (i > 0) load_run<V>(F.u + c - plane, up);
        }
        if (F.vc)
        {
            load_run<V>(F.v + c, v);
            if (j > 0) load_run<V>(F.v + c - d.nz, vp);
        }
        if (F.wc)
        {
            load_run<V>(F.w + c, w);
            if (k > 0)
                wp = __ldg(F.w + c - 1);
            else if (F.ground)
                g = __ldg(F.ground + c / d.nz);
        }
        if (F.uc)
        {
            if (i > 0)
#pragma unroll
                for (int t = 0; t < V; ++t) u[t] = face_mean(up[t], u[t]);
            store_run<V>(F.uc + c, u);
        }
        if (F.vc)
        {
            if (j > 0)
#pragma unroll
                for (int t = 0; t < V; ++t) v[t] = face_mean(vp[t], v[t]);
            store_run<V>(F.vc + c, v);
        }
        if (F.wc)
        {
            float o[V];
            o[0] = k > 0 ? face_mean(wp, w[0]) : __double2float_rn(__dmul_rn(0.5, __dadd_rn(g, (double)w[0])));
#pragma unroll
            for (int t = 1; t < V; ++t) o[t] = face_mean(w[t - 1], w[t]);
            store_run<V>(F.wc + c, o);
        }
    }
}

}  // namespace nimbus
