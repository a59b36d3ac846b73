/*
 * Test infrastructure, not product code: a CPU restatement of the reference
 * Nimbus hot path (split-explicit acoustic loop and conservative WENO5 scalar
 * transport on the flat Cartesian C-grid).  Only tests/, the smoke check and
 * the CPU-baseline leg of bench.py load it, and only as the checker.
 *
 * Built twice from this one source (oracle/oracle.mk):
 *   REAL=float   FP32 storage with FP64 interior arithmetic, the exact
 *                arithmetic sequence of the reference CPU solver; pinned
 *                bit-for-bit against the reference's own objects
 *                (oracle/ref_harness.cpp) by tests/test_oracle_pin.py.
 *   REAL=double  FP64 storage and arithmetic: the FP64 oracle against which
 *                each output field's max/L2 error is stated.
 *
 * Layout: every field is row-major [nx][ny][nz], k fastest.  C-grid: u[i] is
 * the x-face i+1/2, v[j] the y-face j+1/2, w[k] the z-face k+1/2, scalars at
 * cell centres.
 *
 * Compile with -ffp-contract=off: the reference sequences are unfused.
 */
#include <float.h>
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#include <stdlib.h>

#ifndef REAL
#define REAL float
#endif

/* Face-flux and donor-ratio scratch: float in the reference (its Field3D face
 * scratch), double in the FP64 oracle. */
#ifdef ORACLE_FP64
typedef double flux_t;
#else
typedef float flux_t;
#endif

#define IDX(i, j, k) (((size_t)(i) * (size_t)ny + (size_t)(j)) * (size_t)nz + (size_t)(k))

/* Physical constants: include/core/infra/physical_constants.hpp:15-34. */
static const double kRd = 287.0;
static const double kCp = 1004.0;
static const double kP00 = 100000.0;
/* Clamp bounds: include/core/field/field_bounds.hpp:12-17. */
static const float kPMin = 1000.0f, kPMax = 200000.0f;
static const float kRhoMin = 0.05f, kRhoMax = 2.0f;
static const float kWindH = 180.0f, kWindV = 120.0f;
/* KW78 phase speed: boundary_conditions_cartesian_cgrid.cpp:266. */
static const double kCStar = 30.0;

/* Lateral codes: include/init/config/config_v1.hpp:40-48. */
enum { BC_PERIODIC = 0, BC_RADIATIVE = 1, BC_RIGID = 2, BC_RIGID_SLIP = 3, BC_ZERO_GRADIENT = 4 };
/* Bottom: RigidNoSlip=0, RigidSlip=1.  Top: Rigid=0, RigidWithSponge=1, Open=2. */
enum { BOTTOM_NO_SLIP = 0, BOTTOM_SLIP = 1 };
enum { TOP_RIGID = 0, TOP_SPONGE = 1, TOP_OPEN = 2 };

double oracle_gamma(void) { return kCp / (kCp - kRd); }
int oracle_real_bytes(void) { return (int)sizeof(REAL); }

static double finite_or_zero(double v) { return isfinite(v) ? v : 0.0; }
static double safe_rho(double v) { return (isfinite(v) && v > 1.0e-6) ? v : 1.0; }

/* clamp_value: acoustic_cgrid_fast.cpp:38-43 (std::clamp on the stored type). */
static REAL clamp_store(REAL value, REAL fallback, REAL lo, REAL hi)
{
    if (!isfinite(value)) value = fallback;
    return value < lo ? lo : (hi < value ? hi : value);
}

/*
 * One fused acoustic substep, in place: acoustic_cgrid_fast.cpp:12-219.
 * Pass 1 forms the continuity tendency for 1<=i<=nx-2, 1<=j<=ny-2, all k;
 * pass 2 advances rho, clamps, diagnoses p from the dry EOS; pass 3 applies
 * the new pressure gradient to u,v,w (k<=nz-2 for all three) and clamps.
 * drho (may be NULL) receives the stored FP32 continuity tendency.
 */
void oracle_acoustic_fused(int nx, int ny, int nz, double dx, double dy, double dz,
                           REAL* u, REAL* v, REAL* w, REAL* rho, REAL* p, const REAL* theta,
                           const double* rho0, const double* p0, double dt_small, REAL* drho)
{
    const double inv_dx = 1.0 / dx, inv_dy = 1.0 / dy, inv_dz = 1.0 / dz;
    const double gamma = oracle_gamma();
    const size_t n = (size_t)nx * ny * nz;
    REAL* scratch = drho ? drho : (REAL*)malloc(n * sizeof(REAL));

    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
            {
                double d = 0.0;
                if (i >= 1 && i < nx - 1 && j >= 1 && j < ny - 1)
                {
                    const size_t c = IDX(i, j, k);
                    const double rc = (double)rho[c];
                    const double fxp = 0.5 * (rc + (double)rho[IDX(i + 1, j, k)]) * (double)u[c];
                    const double fxm = 0.5 * ((double)rho[IDX(i - 1, j, k)] + rc) * (double)u[IDX(i - 1, j, k)];
                    const double fyp = 0.5 * (rc + (double)rho[IDX(i, j + 1, k)]) * (double)v[c];
                    const double fym = 0.5 * ((double)rho[IDX(i, j - 1, k)] + rc) * (double)v[IDX(i, j - 1, k)];
                    const double fzp = (k + 1 < nz) ? 0.5 * (rc + (double)rho[IDX(i, j, k + 1)]) * (double)w[c]
                                                    : rc * (double)w[c];
                    const double fzm = (k > 0) ? 0.5 * ((double)rho[IDX(i, j, k - 1)] + rc) * (double)w[IDX(i, j, k - 1)]
                                               : 0.0;
                    d = -((fxp - fxm) * inv_dx + (fyp - fym) * inv_dy + (fzp - fzm) * inv_dz);
                }
                scratch[IDX(i, j, k)] = (REAL)finite_or_zero(d);
            }

    for (size_t c = 0; c < n; ++c)
    {
        const int k = (int)(c % (size_t)nz);
        double rn = (double)rho[c] + (double)scratch[c] * dt_small;
        if (!isfinite(rn) || rn <= 0.0) rn = rho0[k] > 0.1 ? rho0[k] : 0.1;
        const REAL rs = clamp_store((REAL)rn, (REAL)1.0, (REAL)kRhoMin, (REAL)kRhoMax);
        rho[c] = rs;
        double pn = (double)100000.0f;
        const double th = (double)theta[c];
        if (th > 0.0) pn = kP00 * pow((double)rs * kRd * th / kP00, gamma);
        if (!isfinite(pn) || pn <= 0.0) pn = (double)100000.0f;
        p[c] = clamp_store((REAL)pn, (REAL)101325.0f, (REAL)kPMin, (REAL)kPMax);
    }

    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
            {
                const size_t c = IDX(i, j, k);
                REAL du = 0, dv = 0, dw = 0;
                if (i >= 1 && i < nx - 1 && j >= 1 && j < ny - 1 && k < nz - 1)
                {
                    const size_t ip = IDX(i + 1, j, k), jp = IDX(i, j + 1, k), kp = IDX(i, j, k + 1);
                    const double rx = 0.5 * ((double)rho[c] + (double)rho[ip]);
                    const double ry = 0.5 * ((double)rho[c] + (double)rho[jp]);
                    const double rz = 0.5 * ((double)rho[c] + (double)rho[kp]);
                    const double dp0dz = (p0[k + 1] - p0[k]) * inv_dz;
                    du = (REAL)finite_or_zero(-((double)p[ip] - (double)p[c]) * inv_dx / safe_rho(rx));
                    dv = (REAL)finite_or_zero(-((double)p[jp] - (double)p[c]) * inv_dy / safe_rho(ry));
                    dw = (REAL)finite_or_zero(-((((double)p[kp] - (double)p[c]) * inv_dz) - dp0dz) / safe_rho(rz));
                }
                u[c] = clamp_store((REAL)((double)u[c] + (double)du * dt_small), 0, -(REAL)kWindH, (REAL)kWindH);
                v[c] = clamp_store((REAL)((double)v[c] + (double)dv * dt_small), 0, -(REAL)kWindH, (REAL)kWindH);
                w[c] = clamp_store((REAL)((double)w[c] + (double)dw * dt_small), 0, -(REAL)kWindV, (REAL)kWindV);
            }
    if (!drho) free(scratch);
}

/*
 * Retained time-averaged face mass flux, Host precision on a flat C-grid:
 * CartesianCGridTransportContext::accumulate_impl (advection_cartesian.cpp:610-870)
 * with cartesian_mass_flux::{x,y,z}_face (cartesian_mass_flux.hpp:57-75,236-404).
 * M += weight * rho_face * (velocity - frame), an unfused FP64 add rounded to
 * the stored type.  Returns 0, or -1 if a stored flux would be non-finite (the
 * reference throws; the stored value is then left unchanged).
 */
int oracle_accumulate_mass_flux(int nx, int ny, int nz, const REAL* rho, const REAL* u, const REAL* v,
                                const REAL* w, double weight, int top_open, double frame_u, double frame_v,
                                REAL* mfx, REAL* mfy, REAL* mfz)
{
    int ok = 1;
#define OR_STORE(dst, flux)                                                   \
    do {                                                                      \
        const double next_ = (double)(dst) + weight * (flux);                 \
        const REAL stored_ = (REAL)next_;                                     \
        if (isfinite(next_) && isfinite((double)stored_)) (dst) = stored_;    \
        else ok = 0;                                                          \
    } while (0)
    for (int i = 0; i < nx - 1; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
            {
                const size_t f = IDX(i, j, k);
                const double vel = frame_u == 0.0 ? (double)u[f] : (double)u[f] - frame_u;
                const double flux = 0.5 * ((double)rho[f] + (double)rho[IDX(i + 1, j, k)]) * vel;
                OR_STORE(mfx[f], flux);
            }
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny - 1; ++j)
            for (int k = 0; k < nz; ++k)
            {
                const size_t f = IDX(i, j, k);
                const double vel = frame_v == 0.0 ? (double)v[f] : (double)v[f] - frame_v;
                const double flux = 0.5 * ((double)rho[f] + (double)rho[IDX(i, j + 1, k)]) * vel;
                OR_STORE(mfy[f], flux);
            }
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
            {
                const size_t f = IDX(i, j, k);
                double flux;
                if (k == nz - 1)
                    flux = top_open ? (double)rho[f] * (double)w[f] : 0.0;
                else
                    flux = 0.5 * ((double)rho[f] + (double)rho[IDX(i, j, k + 1)]) * (double)w[f];
                OR_STORE(mfz[f], flux);
            }
#undef OR_STORE
    return ok ? 0 : -1;
}

/* KW78 radiative face update: include/dynamics/radiative_face.hpp (four
 * rounded operations in the stored type). */
static REAL kw78_face(REAL previous, REAL phase, REAL gradient, REAL dt_rad, REAL inv_spacing, int negative_outgoing)
{
    if (negative_outgoing ? phase >= 0 : phase <= 0) return previous;
    volatile REAL dt_phase = dt_rad * phase;
    volatile REAL tendency = dt_phase * gradient;
    volatile REAL increment = tendency * inv_spacing;
    return previous - increment;
}

/* seed_radiative_state (boundary_conditions_cartesian_cgrid.cpp:798-822).
 * wave layout: u_west[ny*nz], u_east[ny*nz], v_south[nx*nz], v_north[nx*nz]. */
void oracle_seed_radiation(int nx, int ny, int nz, const REAL* u, const REAL* v, REAL* wave)
{
    const size_t yz = (size_t)ny * nz, xz = (size_t)nx * nz;
    for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k)
        {
            wave[(size_t)j * nz + k] = u[IDX(0, j, k)];
            wave[yz + (size_t)j * nz + k] = u[IDX(nx - 2, j, k)];
        }
    for (int i = 0; i < nx; ++i)
        for (int k = 0; k < nz; ++k)
        {
            wave[2 * yz + (size_t)i * nz + k] = v[IDX(i, 0, k)];
            wave[2 * yz + xz + (size_t)i * nz + k] = v[IDX(i, ny - 2, k)];
        }
}

/*
 * Acoustic-substep boundary closure: apply_boundaries
 * (boundary_conditions_cartesian_cgrid.cpp:884-1187).  Faces in the
 * reference's order W, E, S, N (corner ownership), then the vertical pass.
 * dt_rad > 0 integrates the KW78 radiative faces; dt_rad == 0 only refreshes.
 * bc[6] = {west, east, south, north, bottom, top}.
 */
void oracle_acoustic_bcs(int nx, int ny, int nz, double dx, double dy, REAL* u, REAL* v, REAL* w,
                         REAL* rho, REAL* p, REAL* wave, double dt_rad, const int* bc, double frame_u,
                         double frame_v)
{
    const int radiate = dt_rad > 0.0;
    const REAL dtr = (REAL)dt_rad;
    const REAL inv_dx = dx > 0.0 ? (REAL)1 / (REAL)dx : 0;
    const REAL inv_dy = dy > 0.0 ? (REAL)1 / (REAL)dy : 0;
    const REAL fu = (REAL)frame_u, fv = (REAL)frame_v, cstar = (REAL)kCStar;
    const size_t yz = (size_t)ny * nz, xz = (size_t)nx * nz;
    REAL* u_west = wave;
    REAL* u_east = wave + yz;
    REAL* v_south = wave + 2 * yz;
    REAL* v_north = wave + 2 * yz + xz;

#define COPY_RP(di, dj, si, sj, k)                          \
    do {                                                    \
        rho[IDX(di, dj, k)] = rho[IDX(si, sj, k)];          \
        p[IDX(di, dj, k)] = p[IDX(si, sj, k)];              \
    } while (0)

    { /* West: ghost i=0, wall face u[0]. */
        const int b = bc[0];
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
            {
                if (b == BC_PERIODIC)
                {
                    const int s = nx - 2;
                    u[IDX(0, j, k)] = u[IDX(s, j, k)];
                    v[IDX(0, j, k)] = v[IDX(s, j, k)];
                    w[IDX(0, j, k)] = w[IDX(s, j, k)];
                    COPY_RP(0, j, s, j, k);
                    continue;
                }
                if (b == BC_RADIATIVE)
                {
                    if (radiate)
                    {
                        const size_t n = (size_t)j * nz + k;
                        const REAL up = u_west[n];
                        const REAL phase = up - fu - cstar;
                        const REAL un = kw78_face(up, phase, u[IDX(1, j, k)] - up, dtr, inv_dx, 1);
                        u[IDX(0, j, k)] = un;
                        u_west[n] = un;
                    }
                }
                else if (b == BC_ZERO_GRADIENT)
                    u[IDX(0, j, k)] = u[IDX(1, j, k)];
                else
                    u[IDX(0, j, k)] = fu;
                if (b == BC_RIGID) { v[IDX(0, j, k)] = fv; w[IDX(0, j, k)] = 0; }
                else { v[IDX(0, j, k)] = v[IDX(1, j, k)]; w[IDX(0, j, k)] = w[IDX(1, j, k)]; }
                COPY_RP(0, j, 1, j, k);
            }
    }
    { /* East: ghost i=nx-1, wall face u[nx-2]. */
        const int b = bc[1], g = nx - 1, a = nx - 2;
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
            {
                if (b == BC_PERIODIC)
                {
                    u[IDX(g, j, k)] = u[IDX(1, j, k)];
                    v[IDX(g, j, k)] = v[IDX(1, j, k)];
                    w[IDX(g, j, k)] = w[IDX(1, j, k)];
                    COPY_RP(g, j, 1, j, k);
                    continue;
                }
                if (b == BC_RIGID || b == BC_RIGID_SLIP) u[IDX(a, j, k)] = fu;
                if (b == BC_RADIATIVE && radiate)
                {
                    const size_t n = (size_t)j * nz + k;
                    const REAL up = u_east[n];
                    const REAL phase = up - fu + cstar;
                    const REAL un = kw78_face(up, phase, up - u[IDX(a - 1, j, k)], dtr, inv_dx, 0);
                    u[IDX(a, j, k)] = un;
                    u_east[n] = un;
                }
                else if (b == BC_ZERO_GRADIENT)
                    u[IDX(a, j, k)] = u[IDX(a - 1, j, k)];
                u[IDX(g, j, k)] = (b == BC_RADIATIVE || b == BC_ZERO_GRADIENT) ? u[IDX(a, j, k)] : fu;
                if (b == BC_RIGID) { v[IDX(g, j, k)] = fv; w[IDX(g, j, k)] = 0; }
                else { v[IDX(g, j, k)] = v[IDX(a, j, k)]; w[IDX(g, j, k)] = w[IDX(a, j, k)]; }
                COPY_RP(g, j, a, j, k);
            }
    }
    { /* South: ghost j=0, wall face v[i][0]. */
        const int b = bc[2];
        for (int i = 0; i < nx; ++i)
            for (int k = 0; k < nz; ++k)
            {
                if (b == BC_PERIODIC)
                {
                    const int s = ny - 2;
                    v[IDX(i, 0, k)] = v[IDX(i, s, k)];
                    u[IDX(i, 0, k)] = u[IDX(i, s, k)];
                    w[IDX(i, 0, k)] = w[IDX(i, s, k)];
                    COPY_RP(i, 0, i, s, k);
                    continue;
                }
                if (b == BC_RADIATIVE)
                {
                    if (radiate)
                    {
                        const size_t n = (size_t)i * nz + k;
                        const REAL vp = v_south[n];
                        const REAL phase = vp - fv - cstar;
                        const REAL vn = kw78_face(vp, phase, v[IDX(i, 1, k)] - vp, dtr, inv_dy, 1);
                        v[IDX(i, 0, k)] = vn;
                        v_south[n] = vn;
                    }
                }
                else if (b == BC_ZERO_GRADIENT)
                    v[IDX(i, 0, k)] = v[IDX(i, 1, k)];
                else
                    v[IDX(i, 0, k)] = fv;
                if (b == BC_RIGID) { u[IDX(i, 0, k)] = fu; w[IDX(i, 0, k)] = 0; }
                else { u[IDX(i, 0, k)] = u[IDX(i, 1, k)]; w[IDX(i, 0, k)] = w[IDX(i, 1, k)]; }
                COPY_RP(i, 0, i, 1, k);
            }
    }
    { /* North: ghost j=ny-1, wall face v[i][ny-2]. */
        const int b = bc[3], g = ny - 1, a = ny - 2;
        for (int i = 0; i < nx; ++i)
            for (int k = 0; k < nz; ++k)
            {
                if (b == BC_PERIODIC)
                {
                    v[IDX(i, g, k)] = v[IDX(i, 1, k)];
                    u[IDX(i, g, k)] = u[IDX(i, 1, k)];
                    w[IDX(i, g, k)] = w[IDX(i, 1, k)];
                    COPY_RP(i, g, i, 1, k);
                    continue;
                }
                if (b == BC_RIGID || b == BC_RIGID_SLIP) v[IDX(i, a, k)] = fv;
                if (b == BC_RADIATIVE && radiate)
                {
                    const size_t n = (size_t)i * nz + k;
                    const REAL vp = v_north[n];
                    const REAL phase = vp - fv + cstar;
                    const REAL vn = kw78_face(vp, phase, vp - v[IDX(i, a - 1, k)], dtr, inv_dy, 0);
                    v[IDX(i, a, k)] = vn;
                    v_north[n] = vn;
                }
                else if (b == BC_ZERO_GRADIENT)
                    v[IDX(i, a, k)] = v[IDX(i, a - 1, k)];
                v[IDX(i, g, k)] = (b == BC_RADIATIVE || b == BC_ZERO_GRADIENT) ? v[IDX(i, a, k)] : fv;
                if (b == BC_RIGID) { u[IDX(i, g, k)] = fu; w[IDX(i, g, k)] = 0; }
                else { u[IDX(i, g, k)] = u[IDX(i, a, k)]; w[IDX(i, g, k)] = w[IDX(i, a, k)]; }
                COPY_RP(i, g, i, a, k);
            }
    }
#undef COPY_RP
    /* Vertical: apply_vertical_parallel (:1124-1175). */
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
        {
            if (bc[4] == BOTTOM_NO_SLIP)
            {
                u[IDX(i, j, 0)] = 0;
                v[IDX(i, j, 0)] = 0;
            }
            const int kt = nz - 1, km = nz - 2;
            w[IDX(i, j, kt)] = bc[5] == TOP_OPEN ? w[IDX(i, j, km)] : 0;
            u[IDX(i, j, kt)] = u[IDX(i, j, km)];
            v[IDX(i, j, kt)] = v[IDX(i, j, km)];
        }
}

/*
 * The acoustic loop of one large step in the reference CPU order
 * (split_explicit.cpp:174-260 with dynamics.cpp:4545-4557): seed the KW78
 * history from the post-slow faces; then per substep accumulate the retained
 * mass flux from the pre-substep state (capturing rho_begin on the first),
 * run the fused substep, and close the boundaries with dt_small.
 * mfx/mfy/mfz are zeroed here (CartesianCGridTransportContext::begin).
 */
int oracle_acoustic_loop(int nx, int ny, int nz, double dx, double dy, double dz, REAL* u, REAL* v, REAL* w,
                         REAL* rho, REAL* p, const REAL* theta, const double* rho0, const double* p0,
                         double dt_large, int n_substeps, const int* bc, double frame_u, double frame_v,
                         REAL* mfx, REAL* mfy, REAL* mfz, REAL* rho_begin, REAL* wave)
{
    const size_t n = (size_t)nx * ny * nz;
    const double dt_small = dt_large / n_substeps;
    const double weight = dt_small / dt_large;
    int rc = 0;
    memset(mfx, 0, n * sizeof(REAL));
    memset(mfy, 0, n * sizeof(REAL));
    memset(mfz, 0, n * sizeof(REAL));
    memcpy(rho_begin, rho, n * sizeof(REAL));
    oracle_seed_radiation(nx, ny, nz, u, v, wave);
    for (int s = 0; s < n_substeps; ++s)
    {
        rc |= oracle_accumulate_mass_flux(nx, ny, nz, rho, u, v, w, weight, bc[5] == TOP_OPEN, frame_u, frame_v,
                                          mfx, mfy, mfz);
        oracle_acoustic_fused(nx, ny, nz, dx, dy, dz, u, v, w, rho, p, theta, rho0, p0, dt_small, NULL);
        oracle_acoustic_bcs(nx, ny, nz, dx, dy, u, v, w, rho, p, wave, dt_small, bc, frame_u, frame_v);
    }
    return rc;
}

/* ---------------------------------------------------------------------- */
/* Conservative scalar transport.                                          */
/* ---------------------------------------------------------------------- */

/* WENO5-JS face value, upwind stencil (a,b,c,d,e) = (c-2..c+2):
 * include/numerics/advection/weno5_face.hpp:43-86 (Jiang & Shu 1996, ideal
 * weights 1/10, 6/10, 3/10, p = 2, eps = 1e-6 * max(stencil^2) + 1e-40). */
double oracle_weno5_face(double a, double b, double c, double d, double e)
{
    const double p0 = (1.0 / 3.0) * a - (7.0 / 6.0) * b + (11.0 / 6.0) * c;
    const double p1 = -(1.0 / 6.0) * b + (5.0 / 6.0) * c + (1.0 / 3.0) * d;
    const double p2 = (1.0 / 3.0) * c + (5.0 / 6.0) * d - (1.0 / 6.0) * e;
    const double s0a = a - 2.0 * b + c, s0b = a - 4.0 * b + 3.0 * c;
    const double s1a = b - 2.0 * c + d, s1b = b - d;
    const double s2a = c - 2.0 * d + e, s2b = 3.0 * c - 4.0 * d + e;
    const double b0 = (13.0 / 12.0) * s0a * s0a + 0.25 * s0b * s0b;
    const double b1 = (13.0 / 12.0) * s1a * s1a + 0.25 * s1b * s1b;
    const double b2 = (13.0 / 12.0) * s2a * s2a + 0.25 * s2b * s2b;
    double m = a * a;
    if (b * b > m) m = b * b;
    if (c * c > m) m = c * c;
    if (d * d > m) m = d * d;
    if (e * e > m) m = e * e;
    const double eps = 1.0e-6 * m + 1.0e-40;
    const double a0 = (1.0 / 10.0) / ((eps + b0) * (eps + b0));
    const double a1 = (6.0 / 10.0) / ((eps + b1) * (eps + b1));
    const double a2 = (3.0 / 10.0) / ((eps + b2) * (eps + b2));
    const double sum = a0 + a1 + a2;
    if (!(sum > 0.0) || !isfinite(sum)) return c;
    const double face = (a0 * p0 + a1 * p1 + a2 * p2) / sum;
    return isfinite(face) ? face : c;
}

/* minmod3 / mc_limited_slope: advection_cartesian.cpp:136-170. */
static double minmod3(double a, double b, double c)
{
    if (a > 0.0 && b > 0.0 && c > 0.0) return fmin(a, fmin(b, c));
    if (a < 0.0 && b < 0.0 && c < 0.0) return fmax(a, fmax(b, c));
    return 0.0;
}
double oracle_mc_slope(double qm, double q0, double qp)
{
    const double right = qp - q0, left = q0 - qm;
    return minmod3(0.5 * (right + left), 2.0 * right, 2.0 * left);
}

/* Face value along one axis for face l+1/2 of extent n, stencil accessor q(m). */
static double face_value(const REAL* q, size_t base, size_t stride, int l, int n, double mflux, int weno)
{
#define Q(m) ((double)q[base + (size_t)(m) * stride])
    if (mflux >= 0.0)
    {
        const double q0 = Q(l);
        if (weno && l >= 2 && l + 2 <= n - 1) return oracle_weno5_face(Q(l - 2), Q(l - 1), q0, Q(l + 1), Q(l + 2));
        const double sl = (l >= 1) ? oracle_mc_slope(Q(l - 1), q0, Q(l + 1)) : 0.0;
        return q0 + 0.5 * sl;
    }
    const double q0 = Q(l + 1);
    if (weno && l - 1 >= 0 && l + 3 <= n - 1) return oracle_weno5_face(Q(l + 3), Q(l + 2), q0, Q(l), Q(l - 1));
    const double sl = (l + 1 <= n - 2) ? oracle_mc_slope(Q(l), q0, Q(l + 2)) : 0.0;
    return q0 - 0.5 * sl;
#undef Q
}

/* Positive-definite donor ratio store: conservative_pd_limiter_factor
 * (advection_cartesian.hpp:101-108) for the non-support-preserving path. */
static flux_t pd_factor(double r)
{
#ifdef ORACLE_FP64
    return r;
#endif
    if (!(r > 0.0 && r < 1.0)) return (float)r;
    const float roundoff = 1.0f - 32.0f * FLT_EPSILON;
    const float stored = (float)r;
    return nextafterf(stored * roundoff, 0.0f);
}

/*
 * Conservative flux-form transport of n scalars in place on the retained
 * C-grid context: advect_scalar_conservative_3d_cartesian_impl
 * (advection_cartesian.cpp:1652-2640) on its coupled flat C-grid branch.
 * Faces :1943-2172, positive-definite donor limiter :2174-2240, divergence and
 * recovery phi = (rho_b*phi - dt*div SF) / max(rho_end, 0.05) :2465-2640 on
 * 1<=i<=nx-2, 1<=j<=ny-2, all k.  Scalar fluxes and donor ratios are stored
 * as float, as the reference's face scratch is.
 */
int oracle_scalar_transport(int nx, int ny, int nz, double dx, double dy, double dz, REAL** q,
                            const int* positive_definite, int n_scalars, const REAL* rho_end,
                            const REAL* rho_begin, const REAL* mfx, const REAL* mfy, const REAL* mfz, double dt,
                            int weno, int top_open)
{
    const size_t n = (size_t)nx * ny * nz;
    const double inv_dx = 1.0 / dx, inv_dy = 1.0 / dy, inv_dz = 1.0 / dz;
    const double rho_floor = (double)kRhoMin;
    flux_t* sfx = (flux_t*)calloc(n, sizeof(flux_t));
    flux_t* sfy = (flux_t*)calloc(n, sizeof(flux_t));
    flux_t* sfz = (flux_t*)calloc(n, sizeof(flux_t));
    flux_t* rl = (flux_t*)calloc(n, sizeof(flux_t));
    if (!sfx || !sfy || !sfz || !rl) return -1;
    const int kz_end = top_open ? nz : nz - 1;

    for (int s = 0; s < n_scalars; ++s)
    {
        REAL* qs = q[s];
        const int pd = positive_definite[s] != 0;
        for (int i = 0; i < nx - 1; ++i)
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < nz; ++k)
                {
                    const size_t f = IDX(i, j, k);
                    const double mf = (double)mfx[f];
                    const double phi = face_value(qs, IDX(0, j, k), (size_t)ny * nz, i, nx, mf, weno);
                    sfx[f] = (flux_t)(mf * phi);
                }
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny - 1; ++j)
                for (int k = 0; k < nz; ++k)
                {
                    const size_t f = IDX(i, j, k);
                    const double mf = (double)mfy[f];
                    const double phi = face_value(qs, IDX(i, 0, k), (size_t)nz, j, ny, mf, weno);
                    sfy[f] = (flux_t)(mf * phi);
                }
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < kz_end; ++k)
                {
                    const size_t f = IDX(i, j, k);
                    const double mf = (double)mfz[f];
                    if (k == nz - 1)
                    {
                        sfz[f] = (flux_t)(mf * (double)qs[f]);
                        continue;
                    }
                    const double phi = face_value(qs, IDX(i, j, 0), 1, k, nz, mf, weno);
                    sfz[f] = (flux_t)(mf * phi);
                }
        if (pd)
        {
            for (int i = 0; i < nx; ++i)
                for (int j = 0; j < ny; ++j)
                    for (int k = 0; k < nz; ++k)
                    {
                        const size_t c = IDX(i, j, k);
                        double out = 0.0;
                        if (i <= nx - 2 && sfx[c] > (flux_t)0) out += (double)sfx[c] * inv_dx;
                        if (i >= 1 && sfx[IDX(i - 1, j, k)] < (flux_t)0) out -= (double)sfx[IDX(i - 1, j, k)] * inv_dx;
                        if (j <= ny - 2 && sfy[c] > (flux_t)0) out += (double)sfy[c] * inv_dy;
                        if (j >= 1 && sfy[IDX(i, j - 1, k)] < (flux_t)0) out -= (double)sfy[IDX(i, j - 1, k)] * inv_dy;
                        if ((k <= nz - 2 || (top_open && k == nz - 1)) && sfz[c] > (flux_t)0) out += (double)sfz[c] * inv_dz;
                        if (k >= 1 && sfz[IDX(i, j, k - 1)] < (flux_t)0) out -= (double)sfz[IDX(i, j, k - 1)] * inv_dz;
                        double r = 1.0;
                        if (out > 0.0)
                        {
                            const double qc = (double)qs[c];
                            const double avail = (double)rho_begin[c] * ((qc < 0.0) ? 0.0 : qc) / dt; /* std::max(q, 0.0) */
                            r = avail / out < 1.0 ? avail / out : 1.0;
                        }
                        rl[c] = pd_factor(r);
                    }
        }
#define LIMITED(raw, lo, hi) ((!pd || (raw) == (flux_t)0) ? (double)(raw) : (double)(raw) * (double)((raw) > (flux_t)0 ? rl[lo] : rl[hi]))
        for (int i = 1; i < nx - 1; ++i)
            for (int j = 1; j < ny - 1; ++j)
                for (int k = 0; k < nz; ++k)
                {
                    const size_t c = IDX(i, j, k);
                    const size_t cxm = IDX(i - 1, j, k), cxp = IDX(i + 1, j, k);
                    const size_t cym = IDX(i, j - 1, k), cyp = IDX(i, j + 1, k);
                    const int has_top = k <= nz - 2 || (top_open && k == nz - 1);
                    const double sxp = LIMITED(sfx[c], c, cxp);
                    const double sxm = LIMITED(sfx[cxm], cxm, c);
                    const double syp = LIMITED(sfy[c], c, cyp);
                    const double sym = LIMITED(sfy[cym], cym, c);
                    const double szp = has_top ? LIMITED(sfz[c], c, (k < nz - 1 ? IDX(i, j, k + 1) : c)) : 0.0;
                    const double szm = k >= 1 ? LIMITED(sfz[IDX(i, j, k - 1)], IDX(i, j, k - 1), c) : 0.0;
                    const double re = (double)rho_end[c];
                    const double rb = (double)rho_begin[c];
                    double rho_phi;
                    if (pd)
                    {
                        double outgoing = 0.0, incoming = 0.0;
                        if (sxp >= 0.0) outgoing += sxp * inv_dx; else incoming -= sxp * inv_dx;
                        if (sxm <= 0.0) outgoing -= sxm * inv_dx; else incoming += sxm * inv_dx;
                        if (syp >= 0.0) outgoing += syp * inv_dy; else incoming -= syp * inv_dy;
                        if (sym <= 0.0) outgoing -= sym * inv_dy; else incoming += sym * inv_dy;
                        if (has_top) { if (szp >= 0.0) outgoing += szp * inv_dz; else incoming -= szp * inv_dz; }
                        if (k >= 1) { if (szm <= 0.0) outgoing -= szm * inv_dz; else incoming += szm * inv_dz; }
                        rho_phi = (rb * (double)qs[c] - dt * outgoing) + dt * incoming;
                    }
                    else
                    {
                        const double div = (sxp - sxm) * inv_dx + (syp - sym) * inv_dy + (szp - szm) * inv_dz;
                        rho_phi = rb * (double)qs[c] - dt * div;
                    }
                    const double denom = re > rho_floor ? re : rho_floor;
                    qs[c] = (REAL)(rho_phi / denom);
                }
#undef LIMITED
    }
    free(sfx);
    free(sfy);
    free(sfz);
    free(rl);
    return 0;
}

/* ---------------------------------------------------------------------- */
/* Slow tendencies and the Heun (RK2) slow step.                           */
/* ---------------------------------------------------------------------- */

/* Upwind-biased first derivatives, Wicker & Skamarock (2002):
 * include/numerics/derivatives/derivative_operators.hpp:324-395.  `half` is
 * the distance to the nearer boundary along the axis; the stencil order
 * degrades 5 -> 3 -> 1 near it. */
static double upwind_d(const REAL* f, size_t c, size_t stride, int idx, int n, double a, double inv_d)
{
    const int lo = idx, hi = n - 1 - idx;
    const int half = lo < hi ? lo : hi;
#define F(m) ((double)f[c + (ptrdiff_t)(m) * (ptrdiff_t)stride])
    const double cc = F(0);
    if (half <= 0) return 0.0;
    const double m1 = F(-1), p1 = F(1);
    if (half == 1) return (a >= 0.0) ? (cc - m1) * inv_d : (p1 - cc) * inv_d;
    const double m2 = F(-2), p2 = F(2);
    if (half == 2)
        return (a >= 0.0) ? (2.0 * p1 + 3.0 * cc - 6.0 * m1 + m2) * (inv_d / 6.0)
                          : (-p2 + 6.0 * p1 - 3.0 * cc - 2.0 * m1) * (inv_d / 6.0);
    const double m3 = F(-3), p3 = F(3);
    return (a >= 0.0) ? (-2.0 * m3 + 15.0 * m2 - 60.0 * m1 + 20.0 * cc + 30.0 * p1 - 3.0 * p2) * (inv_d / 60.0)
                      : (2.0 * p3 - 15.0 * p2 + 60.0 * p1 - 20.0 * cc - 30.0 * m1 + 3.0 * m2) * (inv_d / 60.0);
#undef F
}

/*
 * Slow tendencies of the flat C-grid KW scheme:
 * CartesianCGrid3DScheme::compute_slow_tendencies (cartesian_cgrid_3d.cpp:1026-1401)
 * on the stationary flat branch.  du (x-faces), dv (y-faces), dw (z-faces)
 * on 1<=i<=nx-2, 1<=j<=ny-2, 0<=k<=nz-2; dp (centres) on 1<=k<=nz-2; zero
 * elsewhere.  qv/qc/qr may be NULL (no moisture / no loading); the loading
 * sums qc+qr (the other hydrometeor species are absent for Kessler).
 * qv0 enters rounded to FP32 (stored_base_value, cartesian_common.hpp:36-40).
 */
void oracle_slow_tendencies(int nx, int ny, int nz, double dx, double dy, double dz, const REAL* u, const REAL* v,
                            const REAL* w, const REAL* rho, const REAL* p, const REAL* qv, const REAL* qc,
                            const REAL* qr, const double* rho0, const double* qv0, const double* u0,
                            const double* v0, double coriolis_f, double frame_u, double frame_v, REAL* du,
                            REAL* dv, REAL* dw, REAL* dp)
{
    const size_t n = (size_t)nx * ny * nz;
    const size_t SX = (size_t)ny * nz, SY = (size_t)nz;
    const double inv_2dx = 1.0 / (2.0 * dx), inv_2dy = 1.0 / (2.0 * dy), inv_2dz = 1.0 / (2.0 * dz);
    const double inv_dx = 1.0 / dx, inv_dy = 1.0 / dy, inv_dz = 1.0 / dz;
    const double g = 9.81;
    for (size_t c = 0; c < n; ++c) du[c] = dv[c] = dw[c] = dp[c] = 0;
    for (int i = 1; i < nx - 1; ++i)
        for (int j = 1; j < ny - 1; ++j)
            for (int k = 0; k < nz - 1; ++k)
            {
                const size_t c = IDX(i, j, k);
                /* du at the x-face */
                {
                    const double ux = (double)u[c];
                    const double uy = 0.25 * ((double)v[IDX(i, j - 1, k)] + (double)v[c] + (double)v[IDX(i + 1, j - 1, k)] +
                                              (double)v[IDX(i + 1, j, k)]);
                    const double tux = ux - frame_u, tuy = uy - frame_v;
                    const double wx = (k == 0) ? 0.25 * ((double)w[IDX(i, j, 0)] + (double)w[IDX(i + 1, j, 0)])
                                               : 0.25 * ((double)w[IDX(i, j, k - 1)] + (double)w[c] +
                                                         (double)w[IDX(i + 1, j, k - 1)] + (double)w[IDX(i + 1, j, k)]);
                    const double ddx = upwind_d(u, c, SX, i, nx, tux, inv_dx);
                    const double ddy = upwind_d(u, c, SY, j, ny, tuy, inv_dy);
                    const double ddz = (k == 0) ? ((wx >= 0.0) ? 0.0 : ((double)u[IDX(i, j, 1)] - (double)u[IDX(i, j, 0)]) * inv_dz)
                                                : upwind_d(u, c, 1, k, nz, wx, inv_dz);
                    const double v0k = v0 ? v0[k] : 0.0;
                    const double cor = coriolis_f * (uy - v0k);
                    du[c] = (REAL)finite_or_zero(-tux * ddx - tuy * ddy - wx * ddz + cor);
                }
                /* dv at the y-face */
                {
                    const double vy = (double)v[c];
                    const double ux = 0.25 * ((double)u[IDX(i - 1, j, k)] + (double)u[c] + (double)u[IDX(i - 1, j + 1, k)] +
                                              (double)u[IDX(i, j + 1, k)]);
                    const double tvy = vy - frame_v, tux = ux - frame_u;
                    const double wy = (k == 0) ? 0.25 * ((double)w[IDX(i, j, 0)] + (double)w[IDX(i, j + 1, 0)])
                                               : 0.25 * ((double)w[IDX(i, j, k - 1)] + (double)w[c] +
                                                         (double)w[IDX(i, j + 1, k - 1)] + (double)w[IDX(i, j + 1, k)]);
                    const double ddx = upwind_d(v, c, SX, i, nx, tux, inv_dx);
                    const double ddy = upwind_d(v, c, SY, j, ny, tvy, inv_dy);
                    const double ddz = (k == 0) ? ((wy >= 0.0) ? 0.0 : ((double)v[IDX(i, j, 1)] - (double)v[IDX(i, j, 0)]) * inv_dz)
                                                : upwind_d(v, c, 1, k, nz, wy, inv_dz);
                    const double u0k = u0 ? u0[k] : 0.0;
                    const double cor = coriolis_f * (ux - u0k);
                    dv[c] = (REAL)finite_or_zero(-tux * ddx - tvy * ddy - wy * ddz - cor);
                }
                /* dw at the z-face: advection, buoyancy, moisture, loading */
                {
                    const double wz = (double)w[c];
                    const double ux = 0.25 * ((double)u[IDX(i - 1, j, k)] + (double)u[c] + (double)u[IDX(i - 1, j, k + 1)] +
                                              (double)u[IDX(i, j, k + 1)]);
                    const double uy = 0.25 * ((double)v[IDX(i, j - 1, k)] + (double)v[c] + (double)v[IDX(i, j - 1, k + 1)] +
                                              (double)v[IDX(i, j, k + 1)]);
                    const double tux = ux - frame_u, tuy = uy - frame_v;
                    const double ddx = upwind_d(w, c, SX, i, nx, tux, inv_dx);
                    const double ddy = upwind_d(w, c, SY, j, ny, tuy, inv_dy);
                    const double ddz = (k == 0) ? ((wz >= 0.0) ? ((double)w[IDX(i, j, 0)] - 0.0) * inv_dz
                                                               : ((double)w[IDX(i, j, 1)] - (double)w[IDX(i, j, 0)]) * inv_dz)
                                                : upwind_d(w, c, 1, k, nz, wz, inv_dz);
                    const double rho_face = 0.5 * ((double)rho[c] + (double)rho[IDX(i, j, k + 1)]);
                    const double rho_s = safe_rho(rho_face);
                    const double rho0_face = 0.5 * (rho0[k] + rho0[k + 1]);
                    const double buoy = -g * (rho_face - rho0_face) / rho_s;
                    double moist = 0.0;
                    if (qv && qv0)
                    {
                        const double qf = 0.5 * ((double)qv[c] + (double)qv[IDX(i, j, k + 1)]);
                        const double q0f = 0.5 * ((double)(float)qv0[k] + (double)(float)qv0[k + 1]);
                        moist = g * 0.608 * (qf - q0f);
                    }
                    double load = 0.0;
                    if (qc)
                    {
                        const double lo = (double)qc[c] + (double)qr[c] + 0.0 + 0.0 + 0.0 + 0.0;
                        const double hi = (double)qc[IDX(i, j, k + 1)] + (double)qr[IDX(i, j, k + 1)] + 0.0 + 0.0 + 0.0 + 0.0;
                        load = -g * (0.5 * (lo + hi));
                    }
                    dw[c] = (REAL)finite_or_zero(-tux * ddx - tuy * ddy - wz * ddz + buoy + moist + load);
                }
                /* dp at the centre: -u.grad p, centred */
                if (k >= 1)
                {
                    const double uc = 0.5 * ((double)u[c] + (double)u[IDX(i - 1, j, k)]);
                    const double vc = 0.5 * ((double)v[c] + (double)v[IDX(i, j - 1, k)]);
                    const double tuc = uc - frame_u, tvc = vc - frame_v;
                    const double wc = 0.5 * ((double)w[c] + (double)w[IDX(i, j, k - 1)]);
                    const double dpdx = ((double)p[IDX(i + 1, j, k)] - (double)p[IDX(i - 1, j, k)]) * inv_2dx;
                    const double dpdy = ((double)p[IDX(i, j + 1, k)] - (double)p[IDX(i, j - 1, k)]) * inv_2dy;
                    const double dpdz = ((double)p[IDX(i, j, k + 1)] - (double)p[IDX(i, j, k - 1)]) * inv_2dz;
                    dp[c] = (REAL)finite_or_zero(-tuc * dpdx - tvc * dpdy - wc * dpdz);
                }
            }
}

/* apply_slow_tendencies_cpu (dynamics.cpp:2066-2092): x += t * dt in FP64,
 * rounded to the stored type; non-finite tendencies count as zero. */
void oracle_slow_apply(size_t n, REAL* u, REAL* v, REAL* w, REAL* p, const REAL* du, const REAL* dv, const REAL* dw,
                       const REAL* dp, double dt)
{
    for (size_t c = 0; c < n; ++c)
    {
        u[c] = (REAL)((double)u[c] + finite_or_zero((double)du[c]) * dt);
        v[c] = (REAL)((double)v[c] + finite_or_zero((double)dv[c]) * dt);
        w[c] = (REAL)((double)w[c] + finite_or_zero((double)dw[c]) * dt);
        p[c] = (REAL)((double)p[c] + finite_or_zero((double)dp[c]) * dt);
    }
}

/*
 * The Heun slow step of one large step, then its application:
 * prepare_slow_rk2_tendencies (dynamics.cpp:5123-5292) -- k1 at the state,
 * predictor state + dt*k1, k2 at the predictor, tendency 0.5f*(k2 + k1) in
 * the stored type -- followed by the split stepper's apply_slow_tendencies(dt)
 * (split_explicit.cpp:186).  u, v, w, p are advanced in place.
 */
int oracle_slow_rk2_step(int nx, int ny, int nz, double dx, double dy, double dz, REAL* u, REAL* v, REAL* w,
                         const REAL* rho, REAL* p, const REAL* qv, const REAL* qc, const REAL* qr, const double* rho0,
                         const double* qv0, const double* u0, const double* v0, double coriolis_f, double frame_u,
                         double frame_v, double dt)
{
    const size_t n = (size_t)nx * ny * nz;
    REAL* buf = (REAL*)malloc(12 * n * sizeof(REAL));
    if (!buf) return -1;
    REAL *k1u = buf, *k1v = buf + n, *k1w = buf + 2 * n, *k1p = buf + 3 * n;
    REAL *k2u = buf + 4 * n, *k2v = buf + 5 * n, *k2w = buf + 6 * n, *k2p = buf + 7 * n;
    REAL *su = buf + 8 * n, *sv = buf + 9 * n, *sw = buf + 10 * n, *sp = buf + 11 * n;
    oracle_slow_tendencies(nx, ny, nz, dx, dy, dz, u, v, w, rho, p, qv, qc, qr, rho0, qv0, u0, v0, coriolis_f, frame_u,
                           frame_v, k1u, k1v, k1w, k1p);
    memcpy(su, u, n * sizeof(REAL));
    memcpy(sv, v, n * sizeof(REAL));
    memcpy(sw, w, n * sizeof(REAL));
    memcpy(sp, p, n * sizeof(REAL));
    oracle_slow_apply(n, su, sv, sw, sp, k1u, k1v, k1w, k1p, dt);
    oracle_slow_tendencies(nx, ny, nz, dx, dy, dz, su, sv, sw, rho, sp, qv, qc, qr, rho0, qv0, u0, v0, coriolis_f,
                           frame_u, frame_v, k2u, k2v, k2w, k2p);
    for (size_t c = 0; c < n; ++c)
    {
        k2u[c] = (REAL)((REAL)0.5 * (k2u[c] + k1u[c]));
        k2v[c] = (REAL)((REAL)0.5 * (k2v[c] + k1v[c]));
        k2w[c] = (REAL)((REAL)0.5 * (k2w[c] + k1w[c]));
        k2p[c] = (REAL)((REAL)0.5 * (k2p[c] + k1p[c]));
    }
    oracle_slow_apply(n, u, v, w, p, k2u, k2v, k2w, k2p, dt);
    free(buf);
    return 0;
}

/* ---------------------------------------------------------------------- */
/* Kessler warm-rain microphysics.                                         */
/* ---------------------------------------------------------------------- */

/* Constants: include/microphysics/microphysics_base.hpp:1073-1080,
 * src/microphysics/base/fall_speeds.hpp:60-68, kessler.hpp:40-46. */
static const double kT0 = 273.15, kLv = 2.5e6, kCpm = 1004.0, kRv = 461.5, kRdm = 287.0, kP0m = 100000.0;
static const double kQc0 = 1.0e-3, kCauto = 1.0e-3, kCaccr = 2.2, kEvapEff = 1.0, kVtMax = 20.0;
static const double kRainA = 36.34, kRainB = 0.1346, kMinQ = 1.0e-9, kRhoFall = 1.2;

static double dclamp(double v, double lo, double hi) { return v < lo ? lo : (hi < v ? hi : v); }
static double dmax(double a, double b) { return a < b ? b : a; }
static double dmin(double a, double b) { return b < a ? b : a; }

/* thermodynamics.hpp:29-44 */
static double theta_to_temperature(double theta, double p)
{
    if (!isfinite(theta) || !isfinite(p)) return kT0;
    const double th = dclamp(theta, 150.0, 700.0), ps = dclamp(p, 100.0, 200000.0);
    const double T = th * pow(ps / kP0m, kRdm / kCpm);
    return isfinite(T) ? T : kT0;
}

/* thermodynamics.hpp:67-85 (Buck, water at all temperatures) */
static double svp_water(double T)
{
    if (!isfinite(T)) return 0.0;
    T = dclamp(T, 150.0, 400.0);
    const double tc = T - kT0;
    const double value = 611.21 * exp((18.678 - tc / 234.5) * tc / (257.14 + tc));
    return isfinite(value) ? dmax(0.0, value) : 0.0;
}

/* thermodynamics.hpp:106-118 */
double oracle_qvs_water(double T, double p)
{
    const double e = svp_water(T);
    if (!isfinite(e) || !isfinite(p)) return 0.0;
    const double ps = dclamp(p, 100.0, 200000.0);
    const double denom = dmax(ps - e, 1.0);
    return dclamp(0.62198 * e / denom, 0.0, 0.2);
}

static double sat_slope(double temperature, double saturation, double p)
{
    if (!(temperature > 150.0 && temperature < 400.0) || !(saturation > 0.0 && saturation < 0.2)) return 0.0;
    const double pressure = dclamp(p, 100.0, 200000.0);
    const double vapor_pressure = saturation * pressure / (0.62198 + saturation);
    const double tc = temperature - kT0;
    const double denominator = 257.14 + tc;
    const double numerator = (18.678 - tc / 234.5) * tc;
    const double numerator_slope = 18.678 - 2.0 * tc / 234.5;
    const double log_pressure_slope = (numerator_slope * denominator - numerator) / (denominator * denominator);
    return saturation * pressure / dmax(pressure - vapor_pressure, 1.0) * log_pressure_slope;
}

/* Coupled saturation adjustment, bracketed Newton on qv' = qvs(T'):
 * thermodynamics.hpp:282-466. */
double oracle_saturation_adjustment(double T_in, double p, double* qv_io, double* qc_io)
{
    double T = isfinite(T_in) ? dclamp(T_in, 150.0, 400.0) : kT0;
    double qv = isfinite(*qv_io) ? dmax(0.0, *qv_io) : 0.0;
    double qc = isfinite(*qc_io) ? dmax(0.0, *qc_io) : 0.0;
    double qvs = oracle_qvs_water(T, p);
    if (!isfinite(qvs) || qvs < 0.0) qvs = 0.0;
    const double L = kLv / kCpm;
    const double eps8 = 8.0 * DBL_EPSILON;
    if (qv > qvs)
    {
        const double maximum = dmin(qv, dmax(0.0, (400.0 - T) / L));
        double condensed = maximum;
        if (qv - maximum - oracle_qvs_water(T + L * maximum, p) <= 0.0)
        {
            double lower = 0.0, upper = maximum;
            condensed = dclamp((qv - qvs) / (1.0 + L * sat_slope(T, qvs, p)), lower, upper);
            for (int it = 0; it < 10; ++it)
            {
                const double ta = T + L * condensed;
                const double sa = oracle_qvs_water(ta, p);
                const double value = qv - condensed - sa;
                const double scale = dmax(dmax(1.0, fabs(qv)), fabs(sa));
                if (fabs(value) <= eps8 * scale) break;
                if (value > 0.0) lower = condensed;
                else upper = condensed;
                const double derivative = -1.0 - L * sat_slope(ta, sa, p);
                const double candidate = condensed - value / derivative;
                condensed = (candidate > lower && candidate < upper) ? candidate : 0.5 * (lower + upper);
            }
        }
        qv -= condensed;
        qc += condensed;
        T += L * condensed;
    }
    else if (qv < qvs && qc > 0.0)
    {
        const double maximum = dmin(qc, dmax(0.0, (T - 150.0) / L));
        double evaporated = maximum;
        if (qv + maximum - oracle_qvs_water(T - L * maximum, p) >= 0.0)
        {
            double lower = 0.0, upper = maximum;
            evaporated = dclamp((qvs - qv) / (1.0 + L * sat_slope(T, qvs, p)), lower, upper);
            for (int it = 0; it < 10; ++it)
            {
                const double ta = T - L * evaporated;
                const double sa = oracle_qvs_water(ta, p);
                const double value = qv + evaporated - sa;
                const double scale = dmax(dmax(1.0, fabs(qv)), fabs(sa));
                if (fabs(value) <= eps8 * scale) break;
                if (value < 0.0) lower = evaporated;
                else upper = evaporated;
                const double derivative = 1.0 + L * sat_slope(ta, sa, p);
                const double candidate = evaporated - value / derivative;
                evaporated = (candidate > lower && candidate < upper) ? candidate : 0.5 * (lower + upper);
            }
        }
        qc -= evaporated;
        qv += evaporated;
        T -= L * evaporated;
    }
    *qc_io = dmax(0.0, qc);
    *qv_io = dmax(0.0, qv);
    return T;
}

/*
 * KesslerScheme::compute_tendencies on its CPU path (kessler.cpp:103-345,
 * warm rain :346-464, sedimentation :465-520) over the cell domain
 * [i0,i1)x[j0,j1)x[k0,k1) with uniform dz.  Tendencies are zero outside the
 * domain; dtheta is converted from the accumulated temperature tendency at
 * the end (temperature_tendency_to_theta, thermodynamics.hpp:225-236).
 * Storage of the tendencies is FP32 in the reference (float fields).
 */
void oracle_kessler_tendencies(int nx, int ny, int nz, double dz, double dt, const REAL* theta, const REAL* p,
                               const REAL* rho, const REAL* qv, const REAL* qc, const REAL* qr, const int* domain,
                               REAL* dth, REAL* dqv, REAL* dqc, REAL* dqr)
{
    const size_t n = (size_t)nx * ny * nz;
    for (size_t c = 0; c < n; ++c) dth[c] = dqv[c] = dqc[c] = dqr[c] = 0;
    if (!(dt > 0.0) || !isfinite(dt)) return;
    const int i0 = domain[0], i1 = domain[1], j0 = domain[2], j1 = domain[3], k0 = domain[4], k1 = domain[5];
    const double inv_dt = 1.0 / dt;
    const double Lcp = kLv / kCpm;
    REAL* temp = (REAL*)malloc(3 * n * sizeof(REAL));
    REAL* qv_adj = temp + n;
    REAL* qc_adj = temp + 2 * n;
    for (int i = i0; i < i1; ++i)
        for (int j = j0; j < j1; ++j)
            for (int k = k0; k < k1; ++k)
            {
                const size_t c = IDX(i, j, k);
                const REAL tv = (REAL)theta_to_temperature((double)theta[c], (double)p[c]);
                double qvd = (double)qv[c], qcd = (double)qc[c];
                const double T = oracle_saturation_adjustment((double)tv, (double)p[c], &qvd, &qcd);
                temp[c] = (REAL)T;
                qv_adj[c] = (REAL)qvd;
                qc_adj[c] = (REAL)qcd;
                const double dqa = (double)qc_adj[c] - (double)qc[c];
                if (dqa != 0.0)
                {
                    const double rate = dqa * inv_dt;
                    dqc[c] += (REAL)rate;
                    dqv[c] -= (REAL)rate;
                    dth[c] += (REAL)(Lcp * rate);
                }
            }
    for (int i = i0; i < i1; ++i)
        for (int j = j0; j < j1; ++j)
            for (int k = k0; k < k1; ++k)
            {
                const size_t c = IDX(i, j, k);
                const REAL qcv = qc_adj[c], qrv = qr[c], qvv = qv_adj[c], T = temp[c];
                REAL prod = 0;
                if (dt > 0.0 && qcv > 0)
                {
                    const double factor = 1.0 / (1.0 + kCaccr * dt * pow((double)(qrv > 0 ? qrv : 0), 0.875));
                    const double amount = (double)qcv * (1.0 - factor) + factor * kCauto * dt * dmax((double)qcv - kQc0, 0.0);
                    prod = (REAL)(dclamp(amount, 0.0, (double)qcv) / dt);
                    dqc[c] -= prod;
                    dqr[c] += prod;
                }
                if (qrv > 0 || prod > 0)
                {
                    const double pv = (double)p[c], rv = (double)rho[c];
                    const double qvsat = oracle_qvs_water((double)T, pv);
                    if (qvsat > 0.0 && (double)qvv < qvsat && rv > 0.0 && pv > 0.0)
                    {
                        const double qr_av = (double)qrv + (double)prod * dt;
                        const double rcgs = 1.0e-3 * rv;
                        const double rain = rcgs * dmax(qr_av, 0.0);
                        const double vent = (1.6 + 124.9 * pow(rain, 0.2046)) * pow(rain, 0.525);
                        const double resist = 2.55e8 / (pv * qvsat) + 5.4e5;
                        const double raw = kEvapEff * (vent / resist) * ((qvsat - (double)qvv) / (rcgs * qvsat));
                        const double gsat = (kLv * kLv * qvsat) / (kCpm * kRv * dmax((double)T * (double)T, 1.0));
                        const double bound = (qvsat - (double)qvv) / (1.0 + gsat);
                        const double evap = dclamp(raw, 0.0, dmin(bound / dt, qr_av / dt));
                        /* Field3D's element proxy rounds a double operand to float
                         * before the compound add (field3d.hpp:391-397). */
                        dqv[c] += (REAL)(float)evap;
                        dqr[c] -= (REAL)(float)evap;
                        dth[c] -= (REAL)(float)(kLv / kCpm * evap);
                    }
                }
            }
    for (int i = i0; i < i1; ++i)
        for (int j = j0; j < j1; ++j)
            for (int k = k0; k < k1; ++k)
            {
                const size_t c = IDX(i, j, k);
                const double rk = (double)rho[c];
                const double rkm = (k > k0) ? (double)rho[IDX(i, j, k - 1)] : rk;
                const double fall = sqrt(kRhoFall / rk);
                const double recv = rk / rkm;
                const double q = dmax(0.0, (double)qr[c]);
                if (q > 0.0)
                {
                    const double vt0 = (q < kMinQ) ? 0.0 : kRainA * pow(1.0e-3 * rk * q, kRainB);
                    const double vt = dmin(vt0 * fall, kVtMax);
                    const float sed = (float)(vt * q);
                    dqr[c] -= (REAL)((double)sed / dz);
                    if (k > k0) dqr[IDX(i, j, k - 1)] += (REAL)(recv * (double)sed / dz);
                }
            }
    for (int i = i0; i < i1; ++i)
        for (int j = j0; j < j1; ++j)
            for (int k = k0; k < k1; ++k)
            {
                const size_t c = IDX(i, j, k);
                const double dT = (double)(float)dth[c], pv = (double)(float)p[c];
                double r = 0.0;
                if (isfinite(dT) && isfinite(pv))
                {
                    const double ps = dclamp(pv, 100.0, 200000.0);
                    r = dT * pow(kP0m / ps, kRdm / kCpm);
                    if (!isfinite(r)) r = 0.0;
                }
                dth[c] = (REAL)r;
            }
    free(temp);
}

/* Application of the Kessler tendencies over the domain, as the CPU commit
 * of step_microphysics_once does it with radiation, boundary layer and
 * stochastic multipliers off (microphysics_step.cpp:3026-3245):
 *  - a non-finite tendency counts as zero;
 *  - water species: bounded_water_value (:480-515), float(q + dq*dt) clamped
 *    to [0, 0.05], non-finite -> 0;
 *  - theta: theta + clamp(dtheta*dt, -50 K, 50 K) in FP64 (a non-finite sum
 *    keeps theta, or theta0 = 300 K if theta itself is not finite), stored
 *    through clamp_theta_k (field_bounds.hpp:68-71): [200, 700] K,
 *    non-finite -> 300 K.  The theta storage residual is only carried with
 *    radiation on and stays zero here. */
void oracle_kessler_apply(int nx, int ny, int nz, double dt, const int* domain, REAL* theta, REAL* qv, REAL* qc,
                          REAL* qr, const REAL* dth, const REAL* dqv, const REAL* dqc, const REAL* dqr)
{
    for (int i = domain[0]; i < domain[1]; ++i)
        for (int j = domain[2]; j < domain[3]; ++j)
            for (int k = domain[4]; k < domain[5]; ++k)
            {
                const size_t c = IDX(i, j, k);
#define WATER(q, dq)                                                       \
    do {                                                                   \
        const double dqs = isfinite((double)(dq)) ? (double)(dq) : 0.0;    \
        const REAL raw = (REAL)((double)(q) + dqs * dt);                   \
        (q) = !isfinite(raw) ? (REAL)0 : (raw < 0 ? (REAL)0 : ((REAL)0.05f < raw ? (REAL)0.05f : raw)); \
    } while (0)
                WATER(qv[c], dqv[c]);
                WATER(qc[c], dqc[c]);
                WATER(qr[c], dqr[c]);
#undef WATER
                const double told = (double)theta[c];
                const double rate = isfinite((double)dth[c]) ? (double)dth[c] : 0.0;
                double total = rate * dt;
                if (!isfinite(total)) total = 0.0;
                const double limited = total < -50.0 ? -50.0 : (50.0 < total ? 50.0 : total);
                double tn = told + limited;
                if (!isfinite(tn)) tn = isfinite(told) ? told : 300.0;
                const REAL stored = (REAL)tn;
                theta[c] = !isfinite((double)stored) ? (REAL)300.0f
                                                     : (stored < (REAL)200.0f ? (REAL)200.0f
                                                                              : ((REAL)700.0f < stored ? (REAL)700.0f
                                                                                                       : stored));
            }
}

/* EOS pressure re-projection (eos_apply.cpp:50-175 with pressure_fp64,
 * eos_pressure.hpp:30-38): p = clamp(float(p00 (rho R_d theta / p00)^gamma))
 * for every cell.  With qv/qc/qr given (a complete moist state) the cells of
 * the attributed domain (physical_scalar_domain: a one-cell lateral ring
 * dropped when the extent is >= 3, every level) are also checked as the energy
 * attribution does (eos_apply.cpp:139-158): the old pressure finite and
 * positive, qv finite and non-negative, qc + qr (FP64) finite and
 * non-negative; the energy sums themselves are diagnostics and are not formed.
 * Returns -1 (and leaves p unchanged) if any cell is invalid, as the
 * reference throws before publishing. */
static int eos_cell_invalid(size_t nx, size_t ny, size_t nz, size_t c, const REAL* rho, const REAL* theta,
                            const REAL* p, const REAL* qv, const REAL* qc, const REAL* qr, double gamma)
{
    const float r = (float)rho[c], th = (float)theta[c];
    const double diag = kP00 * pow((double)r * kRd * (double)th / kP00, gamma);
    if (!isfinite(r) || !(r > 0.0f) || !isfinite(th) || !(th > 0.0f) || !isfinite(diag) || diag <= 0.0 ||
        !isfinite((double)(float)diag))
        return 1;
    if (!qv) return 0;
    const size_t j = (c / nz) % ny, i = c / (nz * ny);
    const size_t ih = nx >= 3, jh = ny >= 3;
    if (i < ih || i >= nx - ih || j < jh || j >= ny - jh) return 0;
    const float p_old = (float)p[c], q = (float)qv[c];
    const double liquid = (double)(float)qc[c] + (double)(float)qr[c];
    return !isfinite(p_old) || p_old <= 0.0f || !isfinite(q) || q < 0.0f || !isfinite(liquid) || liquid < 0.0;
}

int oracle_eos_projection(int nx, int ny, int nz, const REAL* rho, const REAL* theta, REAL* p, const REAL* qv,
                          const REAL* qc, const REAL* qr)
{
    const double gamma = oracle_gamma();
    const size_t n = (size_t)nx * ny * nz;
    for (size_t c = 0; c < n; ++c)
        if (eos_cell_invalid(nx, ny, nz, c, rho, theta, p, qv, qc, qr, gamma)) return -1;
    for (size_t c = 0; c < n; ++c)
    {
        const double diag = kP00 * pow((double)rho[c] * kRd * (double)theta[c] / kP00, gamma);
        p[c] = clamp_store((REAL)(float)diag, (REAL)101325.0f, (REAL)kPMin, (REAL)kPMax);
    }
    return 0;
}

/* ---- End-of-step sponge (state relaxation) ------------------------------
 * apply_rayleigh_damping then apply_lateral_damping on a flat C-grid level
 * (src/core/infra/rayleigh_damping.cpp:720-1119 upper + w-only passes,
 * 1194-1476 lateral pass; relaxation factor :145-163).  Three passes over the
 * whole grid in the reference's order; each cell's increment factor *
 * (ref - old) is formed in FP64 and added to the stored value as the
 * reference's Field3D proxy adds it (rounded to the storage type, then one
 * storage-type add).  Profiles are the reference runtime's: alpha, upper_w_alpha,
 * w_only_alpha, u_ref, v_ref, theta_ref per level; lateral_alpha by distance
 * from the nearest lateral face.  Returns -1 (fields untouched from that pass
 * on) where the reference would throw. */
static int relax_factor(double alpha, double dt, int implicit_mode, double* out)
{
    if (!isfinite(alpha) || alpha < 0.0 || !isfinite(dt) || dt <= 0.0) return -1;
    const double scaled = alpha * dt;
    if (!isfinite(scaled)) return -1;
    *out = implicit_mode ? scaled / (1.0 + scaled) : -expm1(-scaled);
    return 0;
}

static void relax_add(REAL* x, double delta)
{
    *x = (REAL)(*x + (REAL)delta);
}

int oracle_state_relaxation(int nx, int ny, int nz, REAL* u, REAL* v, REAL* w, REAL* theta,
                            const double* theta_ref, const double* alpha, const double* upper_w_alpha,
                            const double* w_only_alpha, const double* u_ref, const double* v_ref,
                            int lateral_width, const double* lateral_alpha, int do_upper, int do_w_only,
                            int do_lateral, int staggered, int implicit_mode, double dt)
{
    const size_t cells = (size_t)nx * ny * nz;
    if (do_upper)
        for (size_t c = 0; c < cells; ++c)
        {
            const int k = (int)(c % (size_t)nz);
            if (alpha[k] <= 0.0 && upper_w_alpha[k] <= 0.0) continue;
            double f, fw;
            if (relax_factor(alpha[k], dt, implicit_mode, &f)) return -1;
            if (staggered)
            {
                if (relax_factor(upper_w_alpha[k], dt, implicit_mode, &fw)) return -1;
            }
            else fw = f;
            const double u_old = u[c], v_old = v[c], w_old = w[c], th_old = theta[c];
            relax_add(&u[c], f * (u_ref[k] - u_old));
            relax_add(&v[c], f * (v_ref[k] - v_old));
            relax_add(&w[c], fw * (0.0 - w_old));
            relax_add(&theta[c], f * (theta_ref[k] - th_old));
        }
    if (do_w_only)
        for (size_t c = 0; c < cells; ++c)
        {
            const int k = (int)(c % (size_t)nz);
            if (w_only_alpha[k] <= 0.0) continue;
            double fw;
            if (relax_factor(w_only_alpha[k], dt, implicit_mode, &fw)) return -1;
            const double w_old = w[c];
            relax_add(&w[c], fw * (0.0 - w_old));
        }
    if (do_lateral && lateral_width > 0)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
            {
                const int di = i < nx - 1 - i ? i : nx - 1 - i;
                const int dj = j < ny - 1 - j ? j : ny - 1 - j;
                const int dist = di < dj ? di : dj;
                if (dist >= lateral_width) continue;
                double f;
                if (relax_factor(lateral_alpha[dist], dt, implicit_mode, &f)) return -1;
                for (int k = 0; k < nz; ++k)
                {
                    const size_t c = ((size_t)i * ny + j) * nz + k;
                    const double u_old = u[c], v_old = v[c], w_old = w[c], th_old = theta[c];
                    relax_add(&u[c], f * (u_ref[k] - u_old));
                    relax_add(&v[c], f * (v_ref[k] - v_old));
                    relax_add(&w[c], f * (0.0 - w_old));
                    relax_add(&theta[c], f * (theta_ref[k] - th_old));
                }
            }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Cell-centre velocities for output (src/core/output/stagger_interpolation.cpp):
 * u: centre i is the mean of faces i-1 and i, cell 0 keeps face 0 (the west
 * boundary face); v likewise in j; w: centre k > 0 is the mean of faces k-1
 * and k, centre 0 is 0.5 (ground_w + w[0]) formed in FP64 and rounded once,
 * with ground_w the column's lower-face velocity (0 on flat ground).  Interior
 * means are 0.5f * (a + b) in storage precision.  A null output skips that
 * component.  Returns -1 when ground_w holds a non-finite value (the
 * reference's invalid_argument), before anything is written. */
int oracle_cell_centre(int nx, int ny, int nz, const REAL* u, const REAL* v, const REAL* w, REAL* uc, REAL* vc,
                       REAL* wc, const double* ground_w)
{
    if (wc && ground_w)
        for (size_t c = 0; c < (size_t)nx * (size_t)ny; ++c)
            if (!isfinite(ground_w[c])) return -1;
    const REAL half = (REAL)0.5;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
        {
            const double lower = ground_w ? ground_w[(size_t)i * (size_t)ny + (size_t)j] : 0.0;
            for (int k = 0; k < nz; ++k)
            {
                const size_t c = IDX(i, j, k);
                if (uc) uc[c] = i == 0 ? u[c] : half * (u[IDX(i - 1, j, k)] + u[c]);
                if (vc) vc[c] = j == 0 ? v[c] : half * (v[IDX(i, j - 1, k)] + v[c]);
                if (wc) wc[c] = k == 0 ? (REAL)(0.5 * (lower + (double)w[c])) : half * (w[c - 1] + w[c]);
            }
        }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Smagorinsky SGS closure on a flat C-grid (stability correction "none").
 *
 * Neighbours (src/turbulence/base/eddy_viscosity.cpp:69-105): clamped to the
 * allocated range, or on a periodic axis wrapped over the physical rows
 * 1..n-2 (the ghost rows 0 and n-1 never take part). */
static int sgs_prev(int i, int n, int periodic)
{
    if (!periodic) return i > 0 ? i - 1 : 0;
    return i <= 1 ? n - 2 : (i - 1 < n - 2 ? i - 1 : n - 2);
}

static int sgs_next(int i, int n, int periodic)
{
    if (!periodic) return i + 1 < n - 1 ? i + 1 : n - 1;
    return i >= n - 2 ? 1 : (i + 1 > 1 ? i + 1 : 1);
}

typedef struct
{
    int nx, ny, nz, use_h, use_v, px, py;
    double dx, dy;
    const double* dz; /* cell thickness per level */
} sgs_grid;

/* Distance between scalar centres k and k+1 (grid_metric_utils.hpp:157-181). */
static double sgs_dzc(const sgs_grid* g, int k) { return 0.5 * (g->dz[k] + g->dz[k + 1]); }

#define SIDX(i, j, k) (((size_t)(i) * (size_t)G->ny + (size_t)(j)) * (size_t)G->nz + (size_t)(k))

static double sgs_w(const sgs_grid* G, const REAL* w, int i, int j, int k)
{
    return k < 0 ? 0.0 : (double)w[SIDX(i, j, k)];
}

/* Strain-rate square at a scalar centre, each component where it lives on
 * the C-grid and the off-diagonal squares averaged from the four edges
 * (compute_directional_strain_sq_centered, eddy_viscosity.cpp:1253-1400).
 * mode: use_h && use_v "3d", use_h alone "horizontal_only", use_v alone
 * "vertical_only". */
static double sgs_strain_sq(const sgs_grid* G, const REAL* u, const REAL* v, const REAL* w, int i, int j, int k)
{
    const int nx = G->nx, ny = G->ny, nz = G->nz;
    const double dx = G->dx, dy = G->dy, dzk = G->dz[k];
    const int jm = sgs_prev(j, ny, G->py), im = sgs_prev(i, nx, G->px);
    const double s11 = ((double)u[SIDX(i, j, k)] - (double)u[SIDX(im, j, k)]) / dx;
    const double s22 = ((double)v[SIDX(i, j, k)] - (double)v[SIDX(i, jm, k)]) / dy;
    const double s33 = (sgs_w(G, w, i, j, k) - sgs_w(G, w, i, j, k - 1)) / dzk;
    double s12[4];
    const int ie[4] = {im, im, i, i}, je[4] = {jm, j, jm, j};
    for (int e = 0; e < 4; ++e)
    {
        const int ii = ie[e], jj = je[e];
        const int jj1 = sgs_next(jj, ny, G->py), ii1 = sgs_next(ii, nx, G->px);
        const double dudy = ((double)u[SIDX(ii, jj1, k)] - (double)u[SIDX(ii, jj, k)]) / dy;
        const double dvdx = ((double)v[SIDX(ii1, jj, k)] - (double)v[SIDX(ii, jj, k)]) / dx;
        s12[e] = 0.5 * (dudy + dvdx);
    }
    /* xz edges (x-face, z-face) and yz edges (y-face, z-face): {d/dz, d w/dx}. */
    double xz[4][2], yz[4][2];
    const int xi[4] = {im, im, i, i}, yj[4] = {jm, jm, j, j}, ke[4] = {k - 1, k, k - 1, k};
    for (int e = 0; e < 4; ++e)
    {
        const int kk = ke[e];
        if (kk < 0 || kk >= nz - 1)
        {
            xz[e][0] = xz[e][1] = yz[e][0] = yz[e][1] = 0.0;
            continue;
        }
        const double dzc = sgs_dzc(G, kk);
        const int ii = xi[e], ii1 = sgs_next(ii, nx, G->px);
        xz[e][0] = ((double)u[SIDX(ii, j, kk + 1)] - (double)u[SIDX(ii, j, kk)]) / dzc;
        xz[e][1] = (sgs_w(G, w, ii1, j, kk) - sgs_w(G, w, ii, j, kk)) / dx;
        const int jj = yj[e], jj1 = sgs_next(jj, ny, G->py);
        yz[e][0] = ((double)v[SIDX(i, jj, kk + 1)] - (double)v[SIDX(i, jj, kk)]) / dzc;
        yz[e][1] = (sgs_w(G, w, i, jj1, kk) - sgs_w(G, w, i, jj, kk)) / dy;
    }
    const double s12_sq = 0.25 * (s12[0] * s12[0] + s12[1] * s12[1] + s12[2] * s12[2] + s12[3] * s12[3]);
#define SGS_AVG_SQ(a, c) (0.25 * (a[0][c] * a[0][c] + a[1][c] * a[1][c] + a[2][c] * a[2][c] + a[3][c] * a[3][c]))
    if (G->use_h && !G->use_v)
        return 2.0 * (s11 * s11 + s22 * s22) + 4.0 * s12_sq + SGS_AVG_SQ(xz, 1) + SGS_AVG_SQ(yz, 1);
    if (G->use_v && !G->use_h)
        return SGS_AVG_SQ(xz, 0) + SGS_AVG_SQ(yz, 0) + 2.0 * s33 * s33;
#undef SGS_AVG_SQ
    double sym_xz[4], sym_yz[4];
    for (int e = 0; e < 4; ++e)
    {
        const double a = 0.5 * (xz[e][0] + xz[e][1]);
        const double b = 0.5 * (yz[e][0] + yz[e][1]);
        sym_xz[e] = a * a;
        sym_yz[e] = b * b;
    }
    const double s13_sq = 0.25 * (sym_xz[0] + sym_xz[1] + sym_xz[2] + sym_xz[3]);
    const double s23_sq = 0.25 * (sym_yz[0] + sym_yz[1] + sym_yz[2] + sym_yz[3]);
    return 2.0 * (s11 * s11 + s22 * s22 + s33 * s33) + 4.0 * (s12_sq + s13_sq + s23_sq);
}

static double sgs_min(double a, double b) { return b < a ? b : a; } /* std::min */

/* Eddy coefficients of every cell (SmagorinskyScheme::compute_eddy_coefficients,
 * smagorinsky.cpp:494-571): nu = Cs^2 Delta^2 |S| (Delta per level: sqrt(dx dy)
 * or cbrt(dx dy dz), precomputed by the caller as the reference does), capped
 * at nu_max; K_theta = nu / Pr_t, K_q = nu / Sc_t, capped at K_max.  Returns
 * -1 at the first cell whose strain, viscosity or diffusivity is not finite
 * (the reference throws), else 0. */
static int sgs_coefficients(const sgs_grid* G, const REAL* u, const REAL* v, const REAL* w, const double* delta,
                            double Cs, double Pr_t, double Sc_t, double nu_max, double K_max, REAL* nu_t,
                            REAL* K_theta, REAL* K_q)
{
    for (int i = 0; i < G->nx; ++i)
        for (int j = 0; j < G->ny; ++j)
            for (int k = 0; k < G->nz; ++k)
            {
                const double strain = sqrt(sgs_strain_sq(G, u, v, w, i, j, k));
                if (!isfinite(strain) || strain < 0.0) return -1;
                double nu = Cs * Cs * delta[k] * delta[k] * strain * 1.0;
                if (!isfinite(nu)) return -1;
                nu = sgs_min(nu, nu_max);
                const double kt = nu / Pr_t, kq = nu / Sc_t;
                if (!isfinite(kt) || !isfinite(kq)) return -1;
                const size_t c = SIDX(i, j, k);
                nu_t[c] = (REAL)nu;
                K_theta[c] = (REAL)sgs_min(kt, K_max);
                K_q[c] = (REAL)sgs_min(kq, K_max);
            }
    return 0;
}

/* Conservative live-density stress divergence (compute_momentum_diffusion_tendencies,
 * eddy_viscosity.cpp:1532-1948, flat C-grid): du_i/dt = (1/rho_face) d_j (2 mu S_ij)
 * with mu = rho nu, diagonal stresses at centres, off-diagonal ones at edges
 * (mu four-point averaged, thickness-weighted across z), zero shear stress at
 * the ground and the lid.  Cells outside the updated faces are zero. */
static void sgs_momentum(const sgs_grid* G, const REAL* u, const REAL* v, const REAL* w, const REAL* rho,
                         const REAL* nu, REAL* dudt, REAL* dvdt, REAL* dwdt)
{
    const int nx = G->nx, ny = G->ny, nz = G->nz, px = G->px, py = G->py;
    const double dx = G->dx, dy = G->dy;
    const size_t n = (size_t)nx * ny * nz;
    for (size_t c = 0; c < n; ++c) dudt[c] = dvdt[c] = dwdt[c] = (REAL)0;
#define MU(ii, jj, kk) ((double)rho[SIDX(ii, jj, kk)] * (double)nu[SIDX(ii, jj, kk)])
#define U(ii, jj, kk) ((double)u[SIDX(ii, jj, kk)])
#define V(ii, jj, kk) ((double)v[SIDX(ii, jj, kk)])
#define W(ii, jj, kk) sgs_w(G, w, ii, jj, kk)
    /* mu on an xy edge (x-face ii, y-face jj) and on xz / yz edges (z-face kk). */
#define MU_XY(ii, jj, kk) (0.25 * (MU(ii, jj, kk) + MU(sgs_next(ii, nx, px), jj, kk) + MU(ii, sgs_next(jj, ny, py), kk) + \
                                   MU(sgs_next(ii, nx, px), sgs_next(jj, ny, py), kk)))
    double lo, up;
    for (int i = 1; i <= (px ? nx - 2 : nx - 3); ++i)
        for (int j = 1; j <= ny - 2; ++j)
        {
            const int jmm = sgs_prev(j, ny, py), imm = sgs_prev(i, nx, px), ipp = sgs_next(i, nx, px);
            double lower = 0.0;
            for (int k = 0; k < nz - 1; ++k)
            {
                double div = 0.0;
                if (G->use_h)
                {
                    const double s_r = (U(ipp, j, k) - U(i, j, k)) / dx;
                    const double s_l = (U(i, j, k) - U(imm, j, k)) / dx;
                    div += (2.0 * MU(ipp, j, k) * s_r - 2.0 * MU(i, j, k) * s_l) / dx;
                    double t12[2];
                    const int jes[2] = {j, jmm};
                    for (int e = 0; e < 2; ++e)
                    {
                        const int je = jes[e], je1 = sgs_next(je, ny, py);
                        const double s12 = 0.5 * ((U(i, je1, k) - U(i, je, k)) / dy + (V(ipp, je, k) - V(i, je, k)) / dx);
                        t12[e] = 2.0 * MU_XY(i, je, k) * s12;
                    }
                    div += (t12[0] - t12[1]) / dy;
                }
                if (G->use_v)
                {
                    double upper = 0.0;
                    if (k < nz - 1)
                    {
                        const double dudz = (U(i, j, k + 1) - U(i, j, k)) / sgs_dzc(G, k);
                        const double grad = G->use_h ? dudz + (W(ipp, j, k) - W(i, j, k)) / dx : dudz;
                        lo = 0.5 * (MU(i, j, k) + MU(ipp, j, k));
                        up = 0.5 * (MU(i, j, k + 1) + MU(ipp, j, k + 1));
                        const double mu_e = (G->dz[k + 1] * lo + G->dz[k] * up) / (G->dz[k] + G->dz[k + 1]);
                        upper = mu_e * grad;
                    }
                    div += (upper - lower) / G->dz[k];
                    lower = upper;
                }
                dudt[SIDX(i, j, k)] = (REAL)(div / (0.5 * ((double)rho[SIDX(i, j, k)] + (double)rho[SIDX(ipp, j, k)])));
            }
        }
    for (int i = 1; i <= nx - 2; ++i)
        for (int j = 1; j <= (py ? ny - 2 : ny - 3); ++j)
        {
            const int jmm = sgs_prev(j, ny, py), jpp = sgs_next(j, ny, py), imm = sgs_prev(i, nx, px);
            double lower = 0.0;
            for (int k = 0; k < nz - 1; ++k)
            {
                double div = 0.0;
                if (G->use_h)
                {
                    const double s_n = (V(i, jpp, k) - V(i, j, k)) / dy;
                    const double s_s = (V(i, j, k) - V(i, jmm, k)) / dy;
                    div += (2.0 * MU(i, jpp, k) * s_n - 2.0 * MU(i, j, k) * s_s) / dy;
                    double t21[2];
                    const int ies[2] = {i, imm};
                    for (int e = 0; e < 2; ++e)
                    {
                        const int ie = ies[e], ie1 = sgs_next(ie, nx, px);
                        const double s12 = 0.5 * ((U(ie, jpp, k) - U(ie, j, k)) / dy + (V(ie1, j, k) - V(ie, j, k)) / dx);
                        t21[e] = 2.0 * MU_XY(ie, j, k) * s12;
                    }
                    div += (t21[0] - t21[1]) / dx;
                }
                if (G->use_v)
                {
                    const double dvdz = (V(i, j, k + 1) - V(i, j, k)) / sgs_dzc(G, k);
                    const double grad = G->use_h ? dvdz + (W(i, jpp, k) - W(i, j, k)) / dy : dvdz;
                    lo = 0.5 * (MU(i, j, k) + MU(i, jpp, k));
                    up = 0.5 * (MU(i, j, k + 1) + MU(i, jpp, k + 1));
                    const double upper = (G->dz[k + 1] * lo + G->dz[k] * up) / (G->dz[k] + G->dz[k + 1]) * grad;
                    div += (upper - lower) / G->dz[k];
                    lower = upper;
                }
                dvdt[SIDX(i, j, k)] = (REAL)(div / (0.5 * ((double)rho[SIDX(i, j, k)] + (double)rho[SIDX(i, jpp, k)])));
            }
        }
    for (int i = 1; i <= nx - 2; ++i)
        for (int j = 1; j <= ny - 2; ++j)
        {
            const int imm = sgs_prev(i, nx, px), jmm = sgs_prev(j, ny, py);
            double lower = 0.0;
            if (G->use_v) lower = 2.0 * MU(i, j, 0) * ((W(i, j, 0) - W(i, j, -1)) / G->dz[0]);
            for (int k = 0; k < nz - 1; ++k)
            {
                const double dzb = G->dz[k], dzt = G->dz[k + 1], dzd = sgs_dzc(G, k);
                const double mass = 0.5 * ((double)rho[SIDX(i, j, k)] * dzb + (double)rho[SIDX(i, j, k + 1)] * dzt);
                double force = 0.0;
                if (G->use_v)
                {
                    const double t33 = 2.0 * MU(i, j, k + 1) * ((W(i, j, k + 1) - W(i, j, k)) / dzt);
                    force += t33 - lower;
                    lower = t33;
                }
                if (G->use_h)
                {
                    double t31[2], t32[2];
                    const int ies[2] = {i, imm}, jes[2] = {j, jmm};
                    for (int e = 0; e < 2; ++e)
                    {
                        const int ie = ies[e], ie1 = sgs_next(ie, nx, px);
                        const double dwdx = (W(ie1, j, k) - W(ie, j, k)) / dx;
                        const double gx = G->use_v ? (U(ie, j, k + 1) - U(ie, j, k)) / dzd + dwdx : dwdx;
                        lo = 0.5 * (MU(ie, j, k) + MU(ie1, j, k));
                        up = 0.5 * (MU(ie, j, k + 1) + MU(ie1, j, k + 1));
                        t31[e] = (G->dz[k + 1] * lo + G->dz[k] * up) / (G->dz[k] + G->dz[k + 1]) * gx;
                        const int je = jes[e], je1 = sgs_next(je, ny, py);
                        const double dwdy = (W(i, je1, k) - W(i, je, k)) / dy;
                        const double gy = G->use_v ? (V(i, je, k + 1) - V(i, je, k)) / dzd + dwdy : dwdy;
                        lo = 0.5 * (MU(i, je, k) + MU(i, je1, k));
                        up = 0.5 * (MU(i, je, k + 1) + MU(i, je1, k + 1));
                        t32[e] = (G->dz[k + 1] * lo + G->dz[k] * up) / (G->dz[k] + G->dz[k + 1]) * gy;
                    }
                    force += dzd * (t31[0] - t31[1]) / dx;
                    force += dzd * (t32[0] - t32[1]) / dy;
                }
                dwdt[SIDX(i, j, k)] = (REAL)(force / mass);
            }
        }
#undef MU_XY
#undef W
#undef V
#undef U
#undef MU
}

/* Conservative scalar diffusion (compute_scalar_diffusion_tendencies,
 * eddy_viscosity.cpp:1953-2090, flat C-grid): d phi/dt = (1/rho) d_j (rho_face
 * K_face d phi/dx_j), zero flux at the ground and lid; a lateral face that is
 * neither periodic nor open reflects its first physical row (zero flux).
 * open: W, E, S, N. */
static void sgs_scalar(const sgs_grid* G, const int* open, const REAL* rho, const REAL* K, const REAL* phi, REAL* out)
{
    const int nx = G->nx, ny = G->ny, nz = G->nz, px = G->px, py = G->py;
    const size_t n = (size_t)nx * ny * nz;
    for (size_t c = 0; c < n; ++c) out[c] = (REAL)0;
#define TR(ii, jj, kk) ((double)rho[SIDX(ii, jj, kk)] * (double)K[SIDX(ii, jj, kk)])
#define PH(ii, jj, kk) ((double)phi[SIDX(ii, jj, kk)])
    for (int i = 1; i <= nx - 2; ++i)
        for (int j = 1; j <= ny - 2; ++j)
        {
            const int jmm = !py && !open[2] && j == 1 ? j : sgs_prev(j, ny, py);
            const int jpp = !py && !open[3] && j == ny - 2 ? j : sgs_next(j, ny, py);
            const int imm = !px && !open[0] && i == 1 ? i : sgs_prev(i, nx, px);
            const int ipp = !px && !open[1] && i == nx - 2 ? i : sgs_next(i, nx, px);
            for (int k = 0; k < nz; ++k)
            {
                double div = 0.0;
                if (G->use_h)
                {
                    const double fe = 0.5 * (TR(i, j, k) + TR(ipp, j, k)) * (PH(ipp, j, k) - PH(i, j, k)) / G->dx;
                    const double fw = 0.5 * (TR(imm, j, k) + TR(i, j, k)) * (PH(i, j, k) - PH(imm, j, k)) / G->dx;
                    const double fn = 0.5 * (TR(i, j, k) + TR(i, jpp, k)) * (PH(i, jpp, k) - PH(i, j, k)) / G->dy;
                    const double fs = 0.5 * (TR(i, jmm, k) + TR(i, j, k)) * (PH(i, j, k) - PH(i, jmm, k)) / G->dy;
                    div += (fe - fw) / G->dx + (fn - fs) / G->dy;
                }
                if (G->use_v)
                {
                    const double ft = k < nz - 1
                        ? 0.5 * (TR(i, j, k) + TR(i, j, k + 1)) * (PH(i, j, k + 1) - PH(i, j, k)) / sgs_dzc(G, k)
                        : 0.0;
                    const double fb = k > 0
                        ? 0.5 * (TR(i, j, k - 1) + TR(i, j, k)) * (PH(i, j, k) - PH(i, j, k - 1)) / sgs_dzc(G, k - 1)
                        : 0.0;
                    div += (ft - fb) / G->dz[k];
                }
                out[SIDX(i, j, k)] = (REAL)(div / (double)rho[SIDX(i, j, k)]);
            }
        }
#undef PH
#undef TR
}

/* The fused Smagorinsky producer: coefficients, then the momentum, theta and
 * (when qv is given) qv tendencies; dqvdt is zero without qv.  Returns -2
 * when an input violates the reference's field contract (u, v, w finite;
 * theta and rho finite and positive; qv finite and non-negative;
 * validate_scheme_inputs, eddy_viscosity.cpp:1088-1175) and nothing is
 * written, -1 when a coefficient is not finite (the outputs are then
 * partial, as the reference's are when it throws).  Else 0. */
int oracle_smagorinsky(int nx, int ny, int nz, const REAL* u, const REAL* v, const REAL* w, const REAL* theta,
                       const REAL* qv, const REAL* rho, const double* dz, const double* delta, double dx, double dy,
                       int use_h, int use_v, int periodic_x, int periodic_y, const int* open_lateral, double Cs,
                       double Pr_t, double Sc_t, double nu_max, double K_max, REAL* nu_t, REAL* K_theta, REAL* K_q,
                       REAL* dudt, REAL* dvdt, REAL* dwdt, REAL* dthdt, REAL* dqvdt)
{
    const sgs_grid g = {nx, ny, nz, use_h, use_v, periodic_x, periodic_y, dx, dy, dz};
    for (size_t c = 0; c < (size_t)nx * ny * nz; ++c)
        if (!isfinite(u[c]) || !isfinite(v[c]) || !isfinite(w[c]) || !isfinite(theta[c]) || !(theta[c] > 0) ||
            !isfinite(rho[c]) || !(rho[c] > 0) || (qv && (!isfinite(qv[c]) || qv[c] < 0)))
            return -2;
    if (sgs_coefficients(&g, u, v, w, delta, Cs, Pr_t, Sc_t, nu_max, K_max, nu_t, K_theta, K_q) != 0) return -1;
    sgs_momentum(&g, u, v, w, rho, nu_t, dudt, dvdt, dwdt);
    sgs_scalar(&g, open_lateral, rho, K_theta, theta, dthdt);
    if (qv)
        sgs_scalar(&g, open_lateral, rho, K_q, qv, dqvdt);
    else
        for (size_t c = 0; c < (size_t)nx * ny * nz; ++c) dqvdt[c] = (REAL)0;
    return 0;
}

/* sanitize_value (include/core/field/field_bounds.hpp:40-56). */
static REAL sgs_sanitize(REAL x, int repairs, REAL fallback, REAL lo, REAL hi)
{
    if (!repairs) return x;
    if (!isfinite(x)) return fallback;
    return x < lo ? lo : (hi < x ? hi : x);
}

/* Forward-Euler application of the SGS tendencies to every cell
 * (apply_sgs_tendencies_cpu, src/core/orchestration/dynamics/sgs_apply.cpp:436-
 * 956, without the work ledger): x += dt * dx/dt in FP64, rounded to FP32 and
 * clamped (winds to +-wind_h / +-wind_v, theta to [theta_lo, theta_hi], qv to
 * [0, qv_hi]); with repairs on, non-finite tendencies count as zero and a
 * non-finite sum falls back (winds and qv to 0, theta to its old value, else
 * the level's base theta, else theta_ref; a non-finite stored theta to
 * (float) theta_ref).  qv and tke (with dtke_pbl) are optional. */
void oracle_sgs_apply(int nx, int ny, int nz, REAL* u, REAL* v, REAL* w, REAL* theta, REAL* qv, REAL* tke,
                      const REAL* dudt, const REAL* dvdt, const REAL* dwdt, const REAL* dthdt, const REAL* dqvdt,
                      const REAL* dtkedt, const REAL* dtke_pbl, const double* theta0_base, double dt, int repairs,
                      double theta_ref, float theta_lo, float theta_hi, float qv_hi, float wind_h, float wind_v)
{
    const size_t plane = (size_t)nz;
    for (size_t c = 0; c < (size_t)nx * ny * nz; ++c)
    {
        double rates[4] = {(double)dudt[c], (double)dvdt[c], (double)dwdt[c], (double)dthdt[c]};
        for (int r = 0; r < 4; ++r)
            if (repairs && !isfinite(rates[r])) rates[r] = 0.0;
        REAL* fields[3] = {u, v, w};
        for (int r = 0; r < 3; ++r)
        {
            double x = (double)fields[r][c] + rates[r] * dt;
            if (repairs && !isfinite(x)) x = 0.0;
            const REAL lim = (REAL)(r == 2 ? wind_v : wind_h);
            fields[r][c] = sgs_sanitize((REAL)x, repairs, (REAL)0, -lim, lim);
        }
        const double th_old = (double)theta[c];
        double th = th_old + rates[3] * dt;
        if (repairs && !isfinite(th))
            th = isfinite(th_old) ? th_old : (theta0_base ? theta0_base[c % plane] : theta_ref);
        theta[c] = sgs_sanitize((REAL)th, repairs, (REAL)(float)theta_ref, (REAL)theta_lo, (REAL)theta_hi);
        if (qv)
        {
            double rq = (double)dqvdt[c];
            if (repairs && !isfinite(rq)) rq = 0.0;
            double q = (double)qv[c] + rq * dt;
            if (repairs && !isfinite(q)) q = 0.0;
            qv[c] = sgs_sanitize((REAL)q, repairs, (REAL)0, (REAL)0, (REAL)qv_hi);
        }
        if (tke)
        {
            const double old = (double)tke[c];
            double a = (double)dtkedt[c], b = (double)dtke_pbl[c];
            if (repairs && !isfinite(a)) a = 0.0;
            if (repairs && !isfinite(b)) b = 0.0;
            double t = old + (a + b) * dt;
            if (repairs && !isfinite(t)) t = isfinite(old) ? old : 0.0;
            tke[c] = (REAL)(repairs ? (t < 0.0 ? 0.0 : t) : t);
        }
    }
}

/* Compensated (Neumaier) sum of the reference's deterministic reductions
 * (CompensatedSum, include/diagnostics/deterministic_reduction.hpp:28-53). */
typedef struct
{
    double sum, corr;
} sgs_csum;

static void sgs_csum_add(sgs_csum* s, double x)
{
    const double next = s->sum + x;
    if (fabs(s->sum) >= fabs(x))
        s->corr += (s->sum - next) + x;
    else
        s->corr += (x - next) + s->sum;
    s->sum = next;
}

/* Explicit stability limit of one SGS substep (compute_sgs_explicit_stability,
 * src/core/orchestration/dynamics/sgs_apply.cpp:1483-1973) on a flat C-grid
 * whose lateral faces are periodic or closed and whose lid carries no open
 * stress, with the reference's deterministic reductions: each x-slab i of the
 * physical cells sums its momentum power (mass u du/dt, per face, in j-k
 * order) and acceleration norm serially, the slabs merge in increasing i with
 * the compensated sum; theta / qv extrema and their monotonic limits are
 * exact min / max reductions.  Limits carry the 0.9 safety factor.
 * dz: per-level thickness (uniform grids: the reference's scalar dz).
 * out: maximum, momentum-energy, theta-monotonic, qv-monotonic timesteps and
 * the irreversible dissipation power.  Returns -2 for an invalid state (the
 * reference's invalid_argument), -4 for a non-dissipative tendency or a
 * non-positive limit (its runtime_error), else 0. */
int oracle_sgs_stability(int nx, int ny, int nz, const REAL* u, const REAL* v, const REAL* w, const REAL* theta,
                         const REAL* qv, const REAL* rho, const REAL* dudt, const REAL* dvdt, const REAL* dwdt,
                         const REAL* dthdt, const REAL* dqvdt, double dx, double dy, const double* dz, int wrap_x,
                         int wrap_y, double* out)
{
    const sgs_grid gg = {nx, ny, nz, 1, 1, wrap_x, wrap_y, dx, dy, dz};
    const sgs_grid* G = &gg;
    for (int i = 1; i < nx - 1; ++i)
        for (int j = 1; j < ny - 1; ++j)
            for (int k = 0; k < nz; ++k)
            {
                const size_t c = SIDX(i, j, k);
                const double vals[9] = {rho[c], u[c], v[c], w[c], theta[c], dudt[c], dvdt[c], dwdt[c], dthdt[c]};
                for (int q = 0; q < 9; ++q)
                    if (!isfinite(vals[q])) return -2;
                if (vals[0] <= 0.0 || vals[4] <= 0.0) return -2;
                if (qv && (!isfinite(qv[c]) || qv[c] < 0 || !isfinite(dqvdt[c]))) return -2;
            }
    const double area = dx * dy;
    sgs_csum power = {0.0, 0.0}, norm = {0.0, 0.0};
    double th_lo = INFINITY, th_hi = -INFINITY, q_lo = INFINITY, q_hi = -INFINITY;
    for (int i = 1; i < nx - 1; ++i)
    {
        double p = 0.0, a = 0.0, slo = INFINITY, shi = -INFINITY, qlo = INFINITY, qhi = -INFINITY;
        for (int j = 1; j < ny - 1; ++j)
            for (int k = 0; k < nz; ++k)
            {
                if (k < nz - 1)
                {
                    const double vol = area * dz[k];
                    if (wrap_x || i <= nx - 3)
                    {
                        const int i1 = wrap_x && i >= nx - 2 ? 1 : i + 1;
                        const double m = 0.5 * ((double)rho[SIDX(i, j, k)] * vol + (double)rho[SIDX(i1, j, k)] * vol);
                        const double acc = (double)dudt[SIDX(i, j, k)];
                        p += m * (double)u[SIDX(i, j, k)] * acc;
                        a += m * acc * acc;
                    }
                    if (wrap_y || j < ny - 2)
                    {
                        const int j1 = wrap_y && j >= ny - 2 ? 1 : j + 1;
                        const double m = 0.5 * ((double)rho[SIDX(i, j, k)] * vol + (double)rho[SIDX(i, j1, k)] * vol);
                        const double acc = (double)dvdt[SIDX(i, j, k)];
                        p += m * (double)v[SIDX(i, j, k)] * acc;
                        a += m * acc * acc;
                    }
                    const double m = 0.5 * ((double)rho[SIDX(i, j, k)] * vol +
                                            (double)rho[SIDX(i, j, k + 1)] * (area * dz[k + 1]));
                    const double acc = (double)dwdt[SIDX(i, j, k)];
                    p += m * (double)w[SIDX(i, j, k)] * acc;
                    a += m * acc * acc;
                }
                const double th = (double)theta[SIDX(i, j, k)];
                slo = th < slo ? th : slo;
                shi = shi < th ? th : shi;
                if (qv)
                {
                    const double q = (double)qv[SIDX(i, j, k)];
                    qlo = q < qlo ? q : qlo;
                    qhi = qhi < q ? q : qhi;
                }
            }
        sgs_csum_add(&power, p);
        sgs_csum_add(&norm, a);
        th_lo = slo < th_lo ? slo : th_lo;
        th_hi = th_hi < shi ? shi : th_hi;
        q_lo = qlo < q_lo ? qlo : q_lo;
        q_hi = q_hi < qhi ? qhi : q_hi;
    }
    const double linear = power.sum + power.corr, anorm = norm.sum + norm.corr;
    if (!isfinite(linear) || !isfinite(anorm) || anorm < 0.0) return -4;
    double mom = INFINITY, dissipation = 0.0;
    if (anorm > 0.0)
    {
        if (!(linear < 0.0)) return -4;
        dissipation = -linear;
        mom = 0.9 * (-2.0 * linear / anorm);
    }
    double tl = INFINITY, ql = INFINITY;
    for (int i = 1; i < nx - 1; ++i)
        for (int j = 1; j < ny - 1; ++j)
            for (int k = 0; k < nz; ++k)
            {
                const size_t c = SIDX(i, j, k);
                const double th = theta[c], r = dthdt[c];
                double x;
                if (r > 0.0)
                {
                    x = (th_hi - th) / r;
                    tl = x < tl ? x : tl;
                }
                else if (r < 0.0)
                {
                    x = (th - th_lo) / -r;
                    tl = x < tl ? x : tl;
                }
                if (qv)
                {
                    const double q = qv[c], rq = dqvdt[c];
                    if (rq > 0.0)
                    {
                        x = (q_hi - q) / rq;
                        ql = x < ql ? x : ql;
                    }
                    else if (rq < 0.0)
                    {
                        x = (q - q_lo) / -rq;
                        ql = x < ql ? x : ql;
                    }
                }
            }
    double lim[2] = {tl, ql};
    for (int q = 0; q < 2; ++q)
    {
        if (isinf(lim[q]) || lim[q] >= 0.5 * DBL_MAX)
            lim[q] = INFINITY;
        else if (!isfinite(lim[q]) || lim[q] <= 0.0)
            return -4;
        else
            lim[q] = 0.9 * lim[q];
    }
    double best = mom;
    if (lim[0] < best) best = lim[0];
    if (lim[1] < best) best = lim[1];
    if (!(best > 0.0)) return -4;
    out[0] = best;
    out[1] = mom;
    out[2] = lim[0];
    out[3] = lim[1];
    out[4] = dissipation;
    return 0;
}

/* ---- Acoustic substep count, re-derived before every large step ----------
 * The largest sound speed the split-explicit scheme must resolve: the flat
 * Cartesian CFL scan's max sqrt(gamma p / rho) over every cell
 * (src/numerics/runtime.cpp:346-401, the product formed as (gamma*p)/rho),
 * raised to that of the base columns (runtime.cpp:854-870).  Returns -1 when
 * a pressure or density is non-finite or non-positive (the reference throws
 * "CFL scan requires finite wind and positive finite pressure/density"). */
int oracle_max_sound_speed(int nx, int ny, int nz, const REAL* p, const REAL* rho, const double* p0,
                           const double* rho0, double* out)
{
    const double gamma = oracle_gamma();
    double best = 0.0;
    const size_t n = (size_t)nx * (size_t)ny * (size_t)nz;
    for (size_t c = 0; c < n; ++c)
    {
        const double ph = (double)p[c], rh = (double)rho[c];
        if (!isfinite(ph) || ph <= 0.0 || !isfinite(rh) || rh <= 0.0) return -1;
        const double s = sqrt(gamma * ph / rh);
        if (best < s) best = s;
    }
    for (int k = 0; k < nz; ++k)
    {
        const double s = sqrt(gamma * p0[k] / rho0[k]);
        if (best < s) best = s;
    }
    *out = best;
    return 0;
}

/* SplitExplicitScheme::resolve_substep_count
 * (src/numerics/time_stepping/schemes/split_explicit/split_explicit.cpp:67-170)
 * with a positive diagnosed minimum spacing: N = max(requested,
 * max(ceil(dt c_max / (0.5 min_spacing)) + 1, 2)); requested <= 0 means the
 * CFL rule alone.  Returns -1 where the reference throws. */
int oracle_resolve_substeps(double dt_large, double c_max, double min_spacing, int requested)
{
    if (!isfinite(dt_large) || dt_large <= 0.0) return -1;
    if (!isfinite(c_max) || c_max <= 0.0) return -1;
    if (!isfinite(min_spacing) || min_spacing <= 0.0) return -1;
    const double required_real = dt_large * c_max / (0.5 * min_spacing);
    if (!isfinite(required_real) || required_real >= (double)(2147483647 - 1)) return -1;
    int required = (int)ceil(required_real) + 1;
    if (required < 2) required = 2;
    if (requested > 0) return requested > required ? requested : required;
    return required;
}
