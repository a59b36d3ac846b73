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
