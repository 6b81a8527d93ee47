// MPDATA kernels, one stage per kernel (the reference's stage structure).
//   k_mpdata_wind   mpdata_compute_wind     src/physics/adv_mpdata.f90:477-504
//   k_upwind        upwind_advection        src/physics/adv_mpdata.f90:43-103
//   k_pseudo        mpdata_fluxes (+ the x0.5 / x0.5*dz scaling of :378-380)
//                                           src/physics/adv_mpdata.f90:105-252
//   k_fct           flux_limiter + FCT core src/physics/adv_mpdata.f90:254-350,
//                                           src/physics/adv_mpdata_FCT_core.f90:47-116
// These kernels are the staged path; the fused path lives in mpdata_fused.cuh.
#pragma once
#include "common.cuh"

namespace icar {

// Decode a flat thread index over (i in [0,ni), k in [0,nz), j in [0,nj)).
struct Idx3 {
    int i, k, j;
    bool ok;
};
__device__ __forceinline__ Idx3 decode(int ni, int nz, int nj)
{
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    Idx3 r;
    r.i = (int)(t % (size_t)ni);
    size_t rest = t / (size_t)ni;
    r.k = (int)(rest % (size_t)nz);
    r.j = (int)(rest / (size_t)nz);
    r.ok = r.j < nj;
    return r;
}

// U_m, V_m, W_m.  rho is 1 unless advect_density.  Threads cover
// i in [0,nx], k, j in [0,ny].
__global__ void k_mpdata_wind(Geo g, float dx, float dt, int adv_den, const float *__restrict__ u,
                              const float *__restrict__ v, const float *__restrict__ w,
                              const float *__restrict__ rho, const float *__restrict__ ju,
                              const float *__restrict__ jv, const float *__restrict__ jw,
                              float *__restrict__ Um, float *__restrict__ Vm, float *__restrict__ Wm)
{
    Idx3 t = decode(g.nx + 1, g.nz, g.ny + 1);
    if (!t.ok) return;
    const int i = t.i, k = t.k, j = t.j;
    if (j < g.ny) {
        size_t c = ix(g, i, k, j);
        if (i >= 1 && i <= g.nx - 1) {
            float rr = adv_den ? rho[c] : 1.0f;
            float rl = adv_den ? rho[c - 1] : 1.0f;
            Um[c] = u[c] * dt * (rr + rl) * 0.5f * ju[c] / dx;
        } else {
            Um[c] = 0.0f;
        }
        if (i < g.nx) {
            float r0 = adv_den ? rho[c] : 1.0f;
            if (k < g.nz - 1) {
                float r1 = adv_den ? rho[ix(g, i, k + 1, j)] : 1.0f;
                Wm[c] = w[c] * dt * jw[c] * (r1 + r0) * 0.5f;
            } else {
                Wm[c] = w[c] * dt * jw[c] * r0;
            }
        }
    }
    if (i < g.nx) {
        size_t c = ix(g, i, k, j);
        if (j >= 1 && j <= g.ny - 1) {
            float rr = adv_den ? rho[c] : 1.0f;
            float rl = adv_den ? rho[ix(g, i, k, j - 1)] : 1.0f;
            Vm[c] = v[c] * dt * (rr + rl) * 0.5f * jv[c] / dx;
        } else {
            Vm[c] = 0.0f;
        }
    }
}

// One donor-cell pass: qout = qin everywhere, interior columns/rows get the
// flux divergence.  U/V/W are Courant fluxes in the face layouts.
__global__ void k_upwind(Geo g, const float *__restrict__ qin, const float *__restrict__ U,
                         const float *__restrict__ V, const float *__restrict__ W,
                         const float *__restrict__ rho, const float *__restrict__ jaco,
                         const float *__restrict__ dz, float *__restrict__ qout)
{
    Idx3 t = decode(g.nx, g.nz, g.ny);
    if (!t.ok) return;
    const int i = t.i, k = t.k, j = t.j;
    const size_t c = ix(g, i, k, j);
    if (i == 0 || i == g.nx - 1 || j == 0 || j == g.ny - 1) {
        qout[c] = qin[c];
        return;
    }
    const size_t sy = (size_t)g.P * g.nz, sz = (size_t)g.P;
    const float q0 = qin[c];
    float fe = flux1(q0, qin[c + 1], U[c + 1]);
    float fw = flux1(qin[c - 1], q0, U[c]);
    float f3 = flux1(q0, qin[c + sy], V[c + sy]);
    float f4 = flux1(qin[c - sy], q0, V[c]);
    float val = q0 - ((fe - fw) + (f3 - f4)) / (jaco[c] * rho[c]);
    float dzjr = dz[c] * jaco[c] * rho[c];
    if (k > 0 && k < g.nz - 1) {
        float f5t = flux1(q0, qin[c + sz], W[c]);
        float f5b = flux1(qin[c - sz], q0, W[c - sz]);
        val = val - (f5t - f5b) / dzjr;
    } else if (k == 0) {
        float f5t = flux1(q0, qin[c + sz], W[c]);
        val = val - f5t / dzjr;
    } else {
        float f5b = flux1(qin[c - sz], q0, W[c - sz]);
        val = val - (q0 * W[c] - f5b) / dzjr;
    }
    qout[c] = val;
}

// Pseudo-velocities, already scaled as mpdata_advect3d does: u2,v2 x0.5 and
// w2 x0.5*dz.  Thread (i,k,j) owns x-face i (row j), y-face j (column i) and
// the top z-face of cell (i,k,j).  w' = W_m/dz and G = J*rho are formed on the
// fly exactly as the reference's temporaries.
__global__ void k_pseudo(Geo g, const float *__restrict__ q, const float *__restrict__ Um,
                         const float *__restrict__ Vm, const float *__restrict__ Wm,
                         const float *__restrict__ rho, const float *__restrict__ jaco,
                         const float *__restrict__ dz, float *__restrict__ u2, float *__restrict__ v2,
                         float *__restrict__ w2)
{
    Idx3 t = decode(g.nx + 1, g.nz, g.ny + 1);
    if (!t.ok) return;
    const int i = t.i, k = t.k, j = t.j, nx = g.nx, ny = g.ny, nz = g.nz;
    const float e10 = 1e-10f, q4 = 1.0f / 4.0f;
    const size_t sy = (size_t)g.P * g.nz, sz = (size_t)g.P;
    const size_t c = ix(g, i, k, j);
#define G_(cc) (jaco[(cc)] * rho[(cc)])
#define WP(cc) (Wm[(cc)] / dz[(cc)])
    // ---- x face i between cells i-1 and i (row j) ----
    if (j < ny) {
        float out = 0.0f;
        if (i >= 1 && i <= nx - 1) {
            float rx = q[c], lx = q[c - 1];
            float uu = Um[c];
            float Gs = G_(c) + G_(c - 1);
            float denom = rx + lx + e10;
            float val = fabsf(uu) * (1.0f - fabsf(uu) / (0.5f * Gs));
            val = val * (rx - lx) / denom;
            if (j > 0 && j < ny - 1) {  // UxV
                float a = q[c + sy], b = q[c - sy], cc = q[c - 1 + sy], d = q[c - 1 - sy];
                float eq = (a - b + cc - d) / (a + b + cc + d + e10);
                float ev = q4 * (Vm[c] + Vm[c + sy] + Vm[c - 1] + Vm[c - 1 + sy]);
                val = val - 0.5f * uu * ev * eq / Gs;
            }
            if (k > 0 && k < nz - 1) {  // UxW
                float a = q[c + sz], b = q[c - sz], cc = q[c - 1 + sz], d = q[c - 1 - sz];
                float eq = (a - b + cc - d) / (a + b + cc + d + e10);
                float ev = q4 * (WP(c) + WP(c - sz) + WP(c - 1) + WP(c - 1 - sz));
                val = val - 0.5f * uu * ev * eq / Gs;
            }
            out = val * 0.5f;
        }
        u2[c] = out;
    }
    if (i < nx) {
        // ---- y face j between rows j-1 and j (column i) ----
        float out = 0.0f;
        if (j >= 1 && j <= ny - 1) {
            float r = q[c], l = q[c - sy];
            float vv = Vm[c];
            float Gs = G_(c) + G_(c - sy);
            float denom = r + l + e10;
            float val = fabsf(vv) * (1.0f - fabsf(vv) / (0.5f * Gs));
            val = val * (r - l) / denom;
            float ev = 0.0f, eq = 0.0f;
            if (i > 0 && i < nx - 1) {  // VxU
                float A = q[c + 1 - sy], B = q[c - 1], C = q[c + 1], D = q[c - 1 - sy];
                eq = (A - B + C - D) / (C + A + B + D + e10);
                ev = q4 * (Um[c + 1] + Um[c + 1 - sy] + Um[c] + Um[c - sy]);
            }
            val = val - 0.5f * vv * ev * eq / Gs;
            if (k > 0 && k < nz - 1) {  // VxW
                float A = q[c + sz - sy], B = q[c - sz], C = q[c + sz], D = q[c - sz - sy];
                float eq2 = (A - B + C - D) / (A + B + C + D + e10);
                float ev2 = q4 * (WP(c) + WP(c - sz) + WP(c - sy) + WP(c - sz - sy));
                val = val - 0.5f * vv * ev2 * eq2 / Gs;
            }
            out = val * 0.5f;
        }
        v2[c] = out;
        // ---- z face: top of cell (i,k,j) ----
        if (j < ny) {
            float o = 0.0f;
            if (k < nz - 1) {
                float r = q[c + sz], l = q[c];
                float ww = WP(c);
                float Gs = G_(c + sz) + G_(c);
                float denom = r + l + e10;
                float val = fabsf(ww) * (1.0f - fabsf(ww) / (0.5f * Gs));
                val = val * (r - l) / denom;
                float ev = 0.0f, eq = 0.0f;
                if (i > 0 && i < nx - 1) {  // WxU
                    float A = q[c + 1 + sz], B = q[c - 1], C = q[c + 1], D = q[c - 1 + sz];
                    eq = (A - B + C - D) / (C + A + B + D + e10);
                    ev = q4 * (Um[c + 1] + Um[c + 1 + sz] + Um[c] + Um[c + sz]);
                }
                val = val - 0.5f * ww * ev * eq / Gs;
                if (j > 0 && j < ny - 1) {  // WxV
                    float A = q[c + sz + sy], B = q[c - sy], C = q[c + sy], D = q[c + sz - sy];
                    float eq2 = (A - B + C - D) / (C + D + A + B + e10);
                    float ev2 = q4 * (Vm[c] + Vm[c + sz] + Vm[c + sy] + Vm[c + sz + sy]);
                    val = val - 0.5f * ww * ev2 * eq2 / Gs;
                }
                o = val * 0.5f * dz[c];
            }
            w2[c] = o;
        }
    }
#undef G_
#undef WP
}

// ---------------------------------------------------------------------------
// FCT on one line of n cells, stated per face.  The reference's sequential
// loop (adv_mpdata_FCT_core.f90:47-116) carries qmax_i2/fin_i2 from face to
// face; unrolled, every cell c has one bound and one in/out flux sum:
//   qmax(c) = max of q1,l over cells c-1..c+1        (1 <= c <= n-2)
//           = max(q1[0],q1[1],l[0],l[1])             (c = 0)
//           = max(q1[n-2],q1[n-1],l[n-2])            (c = n-1, l[n-1] excluded)
//   fin(c)  = max(0,f[c-1]) - min(0,f[c]),  fout(c) = max(0,f[c]) - min(0,f[c-1])
//   at c = 0:   w lines fin = 0-min(0,f[0]), fout = max(0,f[0]); others 0, 0
//   at c = n-1: w lines fin = fout = max(0,f[n-2]) - min(0,f[n-2]); others 0, 0
// and face m (cells m, m+1) is scaled by min(1, beta_in(m+1), beta_out(m)) when
// U2>0, min(1, beta_in(m), beta_out(m+1)) when U2<0.
// LineQ/LineL/LineU give q1, l at cell c and the unlimited U2 at face m.
// ---------------------------------------------------------------------------
template <typename LQ, typename LL, typename LU>
__device__ __forceinline__ void fct_cell_terms(int n, int c, bool is_w, LQ q1, LL l, LU U2, float &qmax,
                                               float &qmin, float &fin, float &fout)
{
    if (c == 0) {
        qmax = fmax_(fmax_(q1(0), q1(1)), fmax_(l(0), l(1)));
        qmin = fmin_(fmin_(q1(0), q1(1)), fmin_(l(0), l(1)));
    } else if (c == n - 1) {
        qmax = fmax_(fmax_(q1(n - 2), q1(n - 1)), l(n - 2));
        qmin = fmin_(fmin_(q1(n - 2), q1(n - 1)), l(n - 2));
    } else {
        qmax = fmax_(fmax_(fmax_(q1(c - 1), q1(c)), q1(c + 1)), fmax_(fmax_(l(c - 1), l(c)), l(c + 1)));
        qmin = fmin_(fmin_(fmin_(q1(c - 1), q1(c)), q1(c + 1)), fmin_(fmin_(l(c - 1), l(c)), l(c + 1)));
    }
    if (c == 0) {
        if (is_w) {
            float f0 = flux1(q1(0), q1(1), U2(0));
            fin = 0.0f - fmin_(0.0f, f0);
            fout = fmax_(0.0f, f0);
        } else {
            fin = 0.0f;
            fout = 0.0f;
        }
    } else if (c == n - 1) {
        if (is_w) {
            float fl = flux1(q1(n - 2), q1(n - 1), U2(n - 2));
            fin = fmax_(0.0f, fl) - fmin_(0.0f, fl);
            fout = fin;
        } else {
            fin = 0.0f;
            fout = 0.0f;
        }
    } else {
        float fl = flux1(q1(c - 1), q1(c), U2(c - 1));
        float fr = flux1(q1(c), q1(c + 1), U2(c));
        fin = fmax_(0.0f, fl) - fmin_(0.0f, fr);
        fout = fmax_(0.0f, fr) - fmin_(0.0f, fl);
    }
}

template <typename LQ, typename LL, typename LU>
__device__ __forceinline__ float fct_face(int n, int m, bool is_w, LQ q1, LL l, LU U2)
{
    const float e15 = 1e-15f;
    float u = U2(m);
    float qmaxL, qminL, finL, foutL, qmaxR, qminR, finR, foutR;
    fct_cell_terms(n, m, is_w, q1, l, U2, qmaxL, qminL, finL, foutL);
    fct_cell_terms(n, m + 1, is_w, q1, l, U2, qmaxR, qminR, finR, foutR);
    if (u > 0.0f) {
        float beta_out_i = (q1(m) - qminL) / (foutL + e15);
        float beta_in_i2 = (qmaxR - q1(m + 1)) / (finR + e15);
        u = fmin_(fmin_(1.0f, beta_in_i2), beta_out_i) * u;
    } else if (u < 0.0f) {
        float beta_in_i = (qmaxL - q1(m)) / (finL + e15);
        float beta_out_i2 = (q1(m + 1) - qminR) / (foutR + e15);
        u = fmin_(fmin_(1.0f, beta_in_i), beta_out_i2) * u;
    }
    return u;
}

// Limit every pseudo-velocity face the reference limits; other faces copy.
// q0 = field before the step (l), q1 = upwind result.  Threads cover
// i in [0,nx], k, j in [0,ny].
__global__ void k_fct(Geo g, const float *__restrict__ q0, const float *__restrict__ q1,
                      const float *__restrict__ u2, const float *__restrict__ v2,
                      const float *__restrict__ w2, float *__restrict__ u2l, float *__restrict__ v2l,
                      float *__restrict__ w2l)
{
    Idx3 t = decode(g.nx + 1, g.nz, g.ny + 1);
    if (!t.ok) return;
    const int i = t.i, k = t.k, j = t.j, nx = g.nx, ny = g.ny, nz = g.nz;
    const size_t sy = (size_t)g.P * g.nz, sz = (size_t)g.P;
    // x face i (between i-1 and i) of row j: limited on rows 1..ny-2
    if (j < ny) {
        const size_t row = ix(g, 0, k, j);
        float out = u2[row + i];
        if (j >= 1 && j <= ny - 2 && i >= 1 && i <= nx - 1) {
            auto Q = [&](int c) { return q1[row + c]; };
            auto L = [&](int c) { return q0[row + c]; };
            auto U = [&](int m) { return u2[row + m + 1]; };
            out = fct_face(nx, i - 1, false, Q, L, U);
        }
        u2l[row + i] = out;
    }
    if (i < nx) {
        // y face j (between j-1 and j) of column i: every column
        const size_t col = ix(g, i, k, 0);
        float out = v2[col + (size_t)j * sy];
        if (j >= 1 && j <= ny - 1) {
            auto Q = [&](int c) { return q1[col + (size_t)c * sy]; };
            auto L = [&](int c) { return q0[col + (size_t)c * sy]; };
            auto U = [&](int m) { return v2[col + (size_t)(m + 1) * sy]; };
            out = fct_face(ny, j - 1, false, Q, L, U);
        }
        v2l[col + (size_t)j * sy] = out;
        // z face: top of cell k; columns 1..nx-2, rows 1..ny-2
        if (j < ny) {
            const size_t zc = ix(g, i, 0, j);
            float o = w2[zc + (size_t)k * sz];
            if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2) {
                if (k == nz - 1) {
                    o = 0.0f;
                } else {
                    auto Q = [&](int c) { return q1[zc + (size_t)c * sz]; };
                    auto L = [&](int c) { return q0[zc + (size_t)c * sz]; };
                    auto U = [&](int m) { return w2[zc + (size_t)m * sz]; };
                    o = fct_face(nz, k, true, Q, L, U);
                }
            }
            w2l[zc + (size_t)k * sz] = o;
        }
    }
}

}  // namespace icar
