// Fused standard-scheme (kADV_STD) advection: one launch per
// adv_std_advect3d call for every species, instead of one kernel per
// reference stage with the flux arrays in HBM.
//
//   k_std_prep    adv_std_compute_wind (advect.f90:447-493) plus the
//                 per-step metric products G = J*rho and DJR = dz*J*rho
//                 (rho = 1 unless advect_density), formed with the
//                 reference's operations so every use is bit-identical.
//   k_std_stage   flux3 + the flux-divergence update (advect.f90:134-251,
//                 298-309) for one RK3 stage or the plain call: out = qold -
//                 div F(qf, t_factor) on the tile, qold elsewhere.
//   k_std_corr    the same with WRF_flux_corr (adv_fluxcorr.f90:37-192):
//                 high-order fluxes, the two half-step upwind fluxes with
//                 the upwind predictor, merged fluxes, per-cell in/out
//                 scale factors and the scaled fluxes, then the update.
//
// Both kernels give one CTA a column tile of one species and march up the
// column.  Horizontally accessed levels (qf, qold, U_m, V_m and, with the
// correction, the predictor and the limiter planes) live in shared-memory
// planes filled by 16-byte cp.async one level ahead; the per-column z state
// (the 6-level window of qf the 5th-order vertical flux needs, the z-face
// fluxes, the scale factors of the cell below, the half-updated value) lives
// in registers, loaded one level ahead of use.
//
// k_std_corr nests three stencils: the update of a tile cell needs the
// scaled fluxes on its faces, hence the scale factors of the cells beside
// it (tile +1), whose in/out sums need the upwind fluxes of the second
// half-step on their faces, hence the predictor on tile +2, whose fluxes
// read qold on tile +3.  Threads own the columns of tile +2 (32 x TY+4); at
// level step b they form the predictor of level b+1 (alpha), the fluxes,
// bounds and scale factors of level b (beta), the horizontal update of
// level b (gamma) and the vertical update of level b-1 (delta), whose top
// face needs the scale factors of level b.
//
// The reference's extended tile (its-1..ite+1) decides where the predictor
// is formed; elsewhere it is qold, as in upwind_flux3's dumb_q.  The
// halo-size rule (order/2 rounded up, +1 with the correction) keeps every
// stencil inside the domain.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"
#include "mpdata_fused.cuh"
#include "std_kernels.cuh"

namespace icar {

__global__ void k_std_prep(Geo g, float dx, float dt, int adv_den, const float *__restrict__ u,
                           const float *__restrict__ v, const float *__restrict__ w, const float *__restrict__ rho,
                           const float *__restrict__ jac, const float *__restrict__ ju, const float *__restrict__ jv,
                           const float *__restrict__ jw, const float *__restrict__ dz, float *__restrict__ Um,
                           float *__restrict__ Vm, float *__restrict__ Wm, float *__restrict__ Gc,
                           float *__restrict__ DJR)
{
    Idx3s t = decode_s(g.nx + 1, g.nz, g.ny + 1);
    if (!t.ok) return;
    const int i = t.i, k = t.k, j = t.j;
    if (j < g.ny) {
        const size_t c = ix(g, i, k, j);
        if (i >= 1 && i <= g.nx - 1) {
            const float rr = adv_den ? rho[c] : 1.0f;
            const float rl = adv_den ? rho[c - 1] : 1.0f;
            Um[c] = u[c] * dt * (rr + rl) * 0.5f * ju[c] / dx;
        } else {
            Um[c] = 0.0f;
        }
        if (i < g.nx) {
            const float r0 = adv_den ? rho[c] : 1.0f;
            if (k < g.nz - 1) {
                const size_t c1 = ix(g, i, k + 1, j);
                const float r1 = adv_den ? rho[c1] : 1.0f;
                const float d0 = dz[c], d1 = dz[c1];
                const float rho_i = (r0 * d0 + r1 * d1) / (d0 + d1);
                Wm[c] = w[c] * dt * jw[c] * rho_i;
            } else {
                Wm[c] = w[c] * dt * jw[c] * r0;
            }
            Gc[c] = jac[c] * r0;
            DJR[c] = dz[c] * jac[c] * r0;
        }
    }
    if (i < g.nx) {
        const size_t c = ix(g, i, k, j);
        if (j >= 1 && j <= g.ny - 1) {
            const float rr = adv_den ? rho[c] : 1.0f;
            const float rl = adv_den ? rho[ix(g, i, k, j - 1)] : 1.0f;
            Vm[c] = v[c] * dt * (rr + rl) * 0.5f * jv[c] / dx;
        } else {
            Vm[c] = 0.0f;
        }
    }
}

// out = qold outside the tile [its,ite] x [jts,jte] (every species of sp:
// q0 = qold, out = out); the fused kernels write only the tile.
__global__ void k_std_ring(Geo g, int hs, const __grid_constant__ SpeciesPtrs sp, int S)
{
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int wx = nx, wy = 2 * hs;                       // rows 0..hs-1 and ny-hs..ny-1, full width
    const int cx = 2 * hs, cy = ny - 2 * hs;              // columns 0..hs-1 and nx-hs..nx-1 of the other rows
    const size_t nrow = (size_t)wx * wy, ncol = (size_t)cx * (cy > 0 ? cy : 0);
    const size_t per = (nrow + ncol) * (size_t)nz;
    const size_t total = per * (size_t)S;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int s = (int)(t / per);
        size_t r = t % per;
        const int k = (int)(r % (size_t)nz);
        r /= (size_t)nz;
        int i, j;
        if (r < nrow) {
            i = (int)(r % (size_t)wx);
            const int jr = (int)(r / (size_t)wx);
            j = jr < hs ? jr : ny - 2 * hs + jr;
        } else {
            r -= nrow;
            const int ir = (int)(r % (size_t)cx);
            j = hs + (int)(r / (size_t)cx);
            i = ir < hs ? ir : nx - 2 * hs + ir;
        }
        if (i < 0 || i >= nx || j < 0 || j >= ny) continue;
        const size_t c = ix(g, i, k, j);
        sp.out[s][c] = sp.q0[s][c];
    }
}

namespace stdf {
// Tile geometry.  CORR: TX = 28 tile columns, threads own the 32 columns of
// tile +2 (x = i0-2+lane) and its TY+4 rows; planes span tile +4 (x from
// floor4(i0-4), 40 wide; TY+8 rows).  Plain stage: TX = 32, threads own the
// tile's columns (x = i0+lane) and TY rows; planes span tile +3 (x from
// floor4(i0-3), 44 wide; TY+6 rows).
template <int TY_, int NW_, bool CORR_>
struct Shape {
    static constexpr bool CORR = CORR_;
    static constexpr int TY = TY_;
    static constexpr int NW = NW_;
    static constexpr int NT = 32 * NW_;
    static constexpr int TX = CORR_ ? 28 : 32;
    static constexpr int HX = CORR_ ? 4 : 3;         // plane halo
    static constexpr int RY = CORR_ ? TY_ + 4 : TY_; // owned rows
    static constexpr int RPW = RY / NW_;
    static constexpr int PW = CORR_ ? 40 : 44;
    static constexpr int PH = TY_ + 2 * HX;
    static constexpr int PLANE = PW * PH;
    static_assert(RY % NW_ == 0, "rows per warp must be whole");
};
// plane slots
constexpr int C_QF = 0;   // 2 slots: level b -> C_QF + (b & 1)
constexpr int C_QO = 2;   // 3 slots: level l -> C_QO + l % 3
constexpr int C_U = 5;    // 3 slots
constexpr int C_V = 8;    // 3 slots
constexpr int C_DQ = 11;  // 2 slots: predictor of level l -> C_DQ + (l & 1)
constexpr int C_MX = 13, C_UX = 14, C_MY = 15, C_UY = 16, C_SI = 17, C_SO = 18;
constexpr int C_NPLANES = 19;
constexpr int P_QF = 0, P_U = 2, P_V = 4, P_FX = 6, P_FY = 7;  // plain stage
constexpr int P_NPLANES = 8;
template <class SH>
constexpr size_t smem_bytes() { return (size_t)(SH::CORR ? C_NPLANES : P_NPLANES) * SH::PLANE * sizeof(float); }

__device__ __forceinline__ int floor4(int x) { return x - (x & 3); }
}  // namespace stdf

// One level of a field into a plane (origin ox, oy), in 16-byte chunks that
// are wholly inside a row's pitch or wholly outside the field (zero-filled).
template <class SH>
struct StdPlaneLoader {
    static constexpr int CPR = SH::PW / 4;
    static constexpr int NCH = (CPR * SH::PH + SH::NT - 1) / SH::NT;
    size_t off[NCH];
    int dst[NCH];
    unsigned okc, okv;
    size_t lstride;
    __device__ __forceinline__ StdPlaneLoader(const Geo &g, int ox, int oy) : okc(0u), okv(0u), lstride((size_t)g.P)
    {
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            const int e = threadIdx.x + c * SH::NT;
            dst[c] = -1;
            off[c] = 0;
            if (e < CPR * SH::PH) {
                const int cx = e % CPR, ly = e / CPR;
                const int i = ox + 4 * cx, j = oy + ly;
                dst[c] = ly * SH::PW + 4 * cx;
                const bool in = i >= 0 && i < g.P && j >= 0;
                if (in && j < g.ny) okc |= 1u << c;
                if (in && j <= g.ny) {
                    okv |= 1u << c;
                    off[c] = (size_t)i + (size_t)g.P * g.nz * j;
                }
            }
        }
    }
    __device__ __forceinline__ void load(float *plane, const float *__restrict__ src, int lev, bool yface) const
    {
        const unsigned ok = yface ? okv : okc;
        const size_t lo = (size_t)lev * lstride;
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            if (dst[c] < 0) continue;
            const bool v = (ok >> c) & 1u;
            cp_async16(plane + dst[c], v ? src + off[c] + lo : src, v);
        }
    }
};

// flux3's vertical flux at face f (bottom face of cell f) from the window
// Q[m] = qf(f-3+m), m = 0..5; ww = W_m(f-1)*t_factor (advect.f90:188-248).
template <int VORD>
__device__ __forceinline__ float std_zflux(int f, int nz, const float *Q, float ww)
{
    if (f == 0) return 0.0f;
    if (f == nz) return Q[2] * ww;
    const bool hi = (VORD == 3 || VORD == 5) && f >= 2 && f <= nz - 2;
    if (VORD == 1 || !hi) return flux1(Q[2], Q[3], ww);
    float F;
    if (VORD == 3 || f == 2 || f == nz - 2) {
        F = 7.0f * (Q[3] + Q[2]) - (Q[4] + Q[1]);
        F = div12(ww * F);
        F = F - div12(fabsf(ww)) * (3.0f * (Q[3] - Q[2]) - (Q[4] - Q[1]));
    } else {
        F = 37.0f * (Q[3] + Q[2]) - 8.0f * (Q[4] + Q[1]) + (Q[5] + Q[0]);
        F = div60(ww * F);
        F = F - div60(fabsf(ww)) * (10.0f * (Q[3] - Q[2]) - 5.0f * (Q[4] - Q[1]) + (Q[5] - Q[0]));
    }
    return F;
}

// Scaled merged flux at a face between cell L (before) and cell R (after),
// adv_fluxcorr.f90:119-135.
__device__ __forceinline__ float wrf_scaled(float F, float si_r, float so_l, float so_r, float si_l)
{
    if (F > 0.0f) return fmin_(si_r, so_l) * F;
    if (F < 0.0f) return fmin_(so_r, si_l) * F;
    return F;
}

// Load helper for the per-column registers: field value at (x, lev, y) of
// an owned column, 0 when the column or level is outside the field.
__device__ __forceinline__ float col_ld(const float *__restrict__ f, size_t c0, size_t P, int lev, int nz, bool ok)
{
    return (ok && lev >= 0 && lev < nz) ? f[c0 + (size_t)lev * P] : 0.0f;
}

// --------------------------------------------------------------------------
// plain stage: out = qold - div F(qf) on the tile
// --------------------------------------------------------------------------
template <int HORD, int VORD, class SH>
__device__ __forceinline__ void std_stage_tile(float *sm, const Geo &g, int its, int ite, int jts, int jte,
                                               float tf, const float *__restrict__ qf,
                                               const float *__restrict__ qold, float *__restrict__ out, int i0,
                                               int j0, const float *__restrict__ Um, const float *__restrict__ Vm,
                                               const float *__restrict__ Wm, const float *__restrict__ Gc,
                                               const float *__restrict__ DJR)
{
    using namespace stdf;
    constexpr int PW = SH::PW, PLANE = SH::PLANE, RPW = SH::RPW, TX = SH::TX, TY = SH::TY;
    const int nz = g.nz;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ox = floor4(i0 - SH::HX), oy = j0 - SH::HX;
    const size_t P = (size_t)g.P;
    auto PL = [&](int slot) { return sm + (size_t)slot * PLANE; };

    const StdPlaneLoader<SH> pl(g, ox, oy);
    pl.load(PL(P_QF), qf, 0, false);
    pl.load(PL(P_U), Um, 0, false);
    pl.load(PL(P_V), Vm, 0, true);
    cp_async_commit();

    const int x = i0 + lane;
    const bool xin = x >= its && x <= ite;
    int yr[RPW];
    bool act[RPW];
    size_t c0[RPW];
    float qfz[RPW][6], wz[RPW], gz[RPW], djr[RPW], qo[RPW], fzb[RPW];
#pragma unroll
    for (int rr = 0; rr < RPW; rr++) {
        yr[rr] = j0 + warp * RPW + rr;
        act[rr] = xin && yr[rr] >= jts && yr[rr] <= jte;
        c0[rr] = act[rr] ? ix(g, x, 0, yr[rr]) : 0;
        qfz[rr][0] = qfz[rr][1] = 0.0f;
#pragma unroll
        for (int m = 2; m < 6; m++) qfz[rr][m] = col_ld(qf, c0[rr], P, m - 2, nz, act[rr]);
        wz[rr] = col_ld(Wm, c0[rr], P, 0, nz, act[rr]);
        gz[rr] = col_ld(Gc, c0[rr], P, 0, nz, act[rr]);
        djr[rr] = col_ld(DJR, c0[rr], P, 0, nz, act[rr]);
        qo[rr] = col_ld(qold, c0[rr], P, 0, nz, act[rr]);
        fzb[rr] = 0.0f;
    }

    for (int b = 0; b < nz; b++) {
        cp_async_wait<0>();
        __syncthreads();
        if (b + 1 < nz) {
            const int s1 = (b + 1) & 1;
            pl.load(PL(P_QF + s1), qf, b + 1, false);
            pl.load(PL(P_U + s1), Um, b + 1, false);
            pl.load(PL(P_V + s1), Vm, b + 1, true);
        }
        cp_async_commit();
        float n_qf[RPW], n_w[RPW], n_g[RPW], n_djr[RPW], n_qo[RPW];
#pragma unroll
        for (int rr = 0; rr < RPW; rr++) {
            n_qf[rr] = col_ld(qf, c0[rr], P, b + 4, nz, act[rr]);
            n_w[rr] = col_ld(Wm, c0[rr], P, b + 1, nz, act[rr]);
            n_g[rr] = col_ld(Gc, c0[rr], P, b + 1, nz, act[rr]);
            n_djr[rr] = col_ld(DJR, c0[rr], P, b + 1, nz, act[rr]);
            n_qo[rr] = col_ld(qold, c0[rr], P, b + 1, nz, act[rr]);
        }
        const float *QF = PL(P_QF + (b & 1));
        const float *U = PL(P_U + (b & 1));
        const float *V = PL(P_V + (b & 1));
        float *FX = PL(P_FX);
        float *FY = PL(P_FY);
        // x faces i0..i0+TX of the tile rows, then y faces j0..j0+TY of the
        // tile columns, as one index range: the leftover faces of both sets
        // share one last partial round instead of one round each.
        constexpr int NFX = (TX + 1) * TY, NF = NFX + TX * (TY + 1);
        for (int e = threadIdx.x; e < NF; e += SH::NT) {
            if (e < NFX) {
                const int fx = e % (TX + 1), ry = e / (TX + 1);
                const int p = (j0 + ry - oy) * PW + (i0 + fx - ox);
                FX[p] = hflux(HORD, QF + p, 1, U[p] * tf);
            } else {
                const int cx = (e - NFX) % TX, fy = (e - NFX) / TX;
                const int p = (j0 + fy - oy) * PW + (i0 + cx - ox);
                FY[p] = hflux(HORD, QF + p, PW, V[p] * tf);
            }
        }
        __syncthreads();
#pragma unroll
        for (int rr = 0; rr < RPW; rr++) {
            const int px = x - ox, py = yr[rr] - oy;
            const int p = py * PW + px;
            const float fzt = std_zflux<VORD>(b + 1, nz, qfz[rr], wz[rr] * tf);
            if (act[rr]) {
                const float tq = qo[rr] - ((FX[p + 1] - FX[p]) + (FY[p + PW] - FY[p])) / gz[rr];
                out[c0[rr] + (size_t)b * P] = tq - (fzt - fzb[rr]) / djr[rr];
            }
            fzb[rr] = fzt;
#pragma unroll
            for (int m = 0; m < 5; m++) qfz[rr][m] = qfz[rr][m + 1];
            qfz[rr][5] = n_qf[rr];
            wz[rr] = n_w[rr];
            gz[rr] = n_g[rr];
            djr[rr] = n_djr[rr];
            qo[rr] = n_qo[rr];
        }
    }
}

// --------------------------------------------------------------------------
// stage with WRF monotonic flux correction
// --------------------------------------------------------------------------
template <int HORD, int VORD, class SH>
__device__ __forceinline__ void std_corr_tile(float *sm, const Geo &g, int its, int ite, int jts, int jte, float tf,
                                              const float *__restrict__ qf, const float *__restrict__ qold,
                                              float *__restrict__ out, int i0, int j0, const float *__restrict__ Um,
                                              const float *__restrict__ Vm, const float *__restrict__ Wm,
                                              const float *__restrict__ Gc, const float *__restrict__ DJR)
{
    using namespace stdf;
    constexpr int PW = SH::PW, PLANE = SH::PLANE, RPW = SH::RPW, TX = SH::TX, TY = SH::TY;
    const int nz = g.nz;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ox = floor4(i0 - SH::HX), oy = j0 - SH::HX;
    const size_t P = (size_t)g.P;
    const float e15 = 1e-15f;
    auto PL = [&](int slot) { return sm + (size_t)slot * PLANE; };

    const StdPlaneLoader<SH> pl(g, ox, oy);
    pl.load(PL(C_QF + 0), qf, 0, false);
    pl.load(PL(C_QO + 0), qold, 0, false);
    pl.load(PL(C_U + 0), Um, 0, false);
    pl.load(PL(C_V + 0), Vm, 0, true);
    if (nz > 1) {
        pl.load(PL(C_QO + 1), qold, 1, false);
        pl.load(PL(C_U + 1), Um, 1, false);
        pl.load(PL(C_V + 1), Vm, 1, true);
    }
    cp_async_commit();

    // owned column: x = i0-2+lane, rows y = j0-2+warp*RPW+rr
    const int x = i0 - 2 + lane;
    const bool xdom = x >= 0 && x < g.nx;
    const bool xext = x >= its - 1 && x <= ite + 1;          // the reference's extended tile
    const bool xE = lane >= 1 && lane <= TX + 2;             // tile +1 (scale factors)
    const bool xT = lane >= 2 && lane <= TX + 1 && x >= its && x <= ite;
    const int px = x - ox;
    int yr[RPW], pr[RPW];
    bool ld[RPW], pext[RPW], isE[RPW], isT[RPW];
    size_t c0[RPW];
    // z state (see the header): windows and carried face values
    float qfz[RPW][6], qoz[RPW][4], wz[RPW][3], gz[RPW][2], dj[RPW][3];
    float dq0[RPW], u1lo[RPW], ufzb[RPW], mzb[RPW], sidn[RPW], sodn[RPW], fzfdn[RPW], tqdn[RPW];
#pragma unroll
    for (int rr = 0; rr < RPW; rr++) {
        const int r = warp * RPW + rr;
        yr[rr] = j0 - 2 + r;
        pr[rr] = (yr[rr] - oy) * PW + px;
        ld[rr] = xdom && yr[rr] >= 0 && yr[rr] < g.ny;
        pext[rr] = xext && yr[rr] >= jts - 1 && yr[rr] <= jte + 1;
        isE[rr] = xE && r >= 1 && r <= TY + 2;
        isT[rr] = xT && r >= 2 && r <= TY + 1 && yr[rr] >= jts && yr[rr] <= jte;
        c0[rr] = ld[rr] ? ix(g, x, 0, yr[rr]) : 0;
        qfz[rr][0] = qfz[rr][1] = 0.0f;
#pragma unroll
        for (int m = 2; m < 6; m++) qfz[rr][m] = col_ld(qf, c0[rr], P, m - 2, nz, ld[rr]);
        qoz[rr][0] = 0.0f;
#pragma unroll
        for (int m = 1; m < 4; m++) qoz[rr][m] = col_ld(qold, c0[rr], P, m - 1, nz, ld[rr]);
        wz[rr][0] = 0.0f;
        wz[rr][1] = col_ld(Wm, c0[rr], P, 0, nz, ld[rr]);
        wz[rr][2] = col_ld(Wm, c0[rr], P, 1, nz, ld[rr]);
        gz[rr][0] = col_ld(Gc, c0[rr], P, 0, nz, ld[rr]);
        gz[rr][1] = col_ld(Gc, c0[rr], P, 1, nz, ld[rr]);
        dj[rr][0] = 1.0f;
        dj[rr][1] = col_ld(DJR, c0[rr], P, 0, nz, ld[rr]);
        dj[rr][2] = col_ld(DJR, c0[rr], P, 1, nz, ld[rr]);
        u1lo[rr] = ufzb[rr] = mzb[rr] = 0.0f;
        sidn[rr] = sodn[rr] = 1.0f;
        fzfdn[rr] = tqdn[rr] = 0.0f;
        dq0[rr] = 0.0f;
    }

    // alpha: upwind predictor of level a (upwind_flux3's dumb_q) for the
    // owned cells, written to its plane; returns the first half-step flux
    // through the top face in u1hi.  qa, qa1 = qold(a), qold(a+1); wa, ga,
    // da = W_m, G, DJR at a; u1b = first half-step flux through face a.
    auto alpha = [&](int a, int rr, float qa, float qa1, float wa, float ga, float da, float u1b, float &u1hi) {
        const float *QO = PL(C_QO + a % 3);
        const float *U = PL(C_U + a % 3);
        const float *V = PL(C_V + a % 3);
        const int p = pr[rr];
        u1hi = a + 1 < nz ? half_up(wa, qa, qa1) : 0.5f * qa * wa;
        float d = qa;
        if (pext[rr]) {
            const float fxl = half_up(U[p], QO[p - 1], qa), fxr = half_up(U[p + 1], qa, QO[p + 1]);
            const float fyl = half_up(V[p], QO[p - PW], qa), fyr = half_up(V[p + PW], qa, QO[p + PW]);
            d = qa - ((fxr - fxl) + (fyr - fyl)) / ga;
            d = d - (u1hi - u1b) / da;
        }
        PL(C_DQ + (a & 1))[p] = d;
        return d;
    };

    cp_async_wait<0>();
    __syncthreads();
#pragma unroll
    for (int rr = 0; rr < RPW; rr++) {
        float hi;
        dq0[rr] = alpha(0, rr, qoz[rr][1], qoz[rr][2], wz[rr][1], gz[rr][0], dj[rr][1], 0.0f, hi);
        u1lo[rr] = hi;
    }

    for (int b = 0; b < nz; b++) {
        cp_async_wait<0>();
        __syncthreads();  // B0
        if (b + 1 < nz) pl.load(PL(C_QF + ((b + 1) & 1)), qf, b + 1, false);
        if (b + 2 < nz) {
            const int s2 = (b + 2) % 3;
            pl.load(PL(C_QO + s2), qold, b + 2, false);
            pl.load(PL(C_U + s2), Um, b + 2, false);
            pl.load(PL(C_V + s2), Vm, b + 2, true);
        }
        cp_async_commit();
        float n_qf[RPW], n_qo[RPW], n_w[RPW], n_g[RPW], n_dj[RPW];
#pragma unroll
        for (int rr = 0; rr < RPW; rr++) {
            n_qf[rr] = col_ld(qf, c0[rr], P, b + 4, nz, ld[rr]);
            n_qo[rr] = col_ld(qold, c0[rr], P, b + 3, nz, ld[rr]);
            n_w[rr] = col_ld(Wm, c0[rr], P, b + 2, nz, ld[rr]);
            n_g[rr] = col_ld(Gc, c0[rr], P, b + 2, nz, ld[rr]);
            n_dj[rr] = col_ld(DJR, c0[rr], P, b + 2, nz, ld[rr]);
        }
        // alpha at level b+1
        float dq1[RPW], u1hi[RPW];
#pragma unroll
        for (int rr = 0; rr < RPW; rr++) {
            dq1[rr] = 0.0f;
            u1hi[rr] = 0.0f;
            if (b + 1 < nz)
                dq1[rr] = alpha(b + 1, rr, qoz[rr][2], qoz[rr][3], wz[rr][2], gz[rr][1], dj[rr][2], u1lo[rr], u1hi[rr]);
        }
        // beta, faces: merged and upwind fluxes on every face of tile +1 at level b
        {
            const float *QF = PL(C_QF + (b & 1));
            const float *QO = PL(C_QO + b % 3);
            const float *U = PL(C_U + b % 3);
            const float *V = PL(C_V + b % 3);
            const float *DQ = PL(C_DQ + (b & 1));
            float *MX = PL(C_MX), *UX = PL(C_UX), *MY = PL(C_MY), *UY = PL(C_UY);
            // x faces i0-1..i0+TX+1 on rows j0-1..j0+TY
            for (int e = threadIdx.x; e < (TX + 3) * (TY + 2); e += SH::NT) {
                const int fx = e % (TX + 3), ry = e / (TX + 3);
                const int p = (j0 - 1 + ry - oy) * PW + (i0 - 1 + fx - ox);
                const float u = U[p];
                const float F = hflux(HORD, QF + p, 1, u * tf);
                const float uf = half_up(u, QO[p - 1], QO[p]) + half_up(u, DQ[p - 1], DQ[p]);
                MX[p] = F - uf;
                UX[p] = uf;
            }
            // y faces j0-1..j0+TY+1 on columns i0-1..i0+TX
            for (int e = threadIdx.x; e < (TX + 2) * (TY + 3); e += SH::NT) {
                const int cx = e % (TX + 2), fy = e / (TX + 2);
                const int p = (j0 - 1 + fy - oy) * PW + (i0 - 1 + cx - ox);
                const float vv = V[p];
                const float F = hflux(HORD, QF + p, PW, vv * tf);
                const float uf = half_up(vv, QO[p - PW], QO[p]) + half_up(vv, DQ[p - PW], DQ[p]);
                MY[p] = F - uf;
                UY[p] = uf;
            }
        }
        // beta, z faces of the owned column: face b+1
        float ufzt[RPW], mzt[RPW];
#pragma unroll
        for (int rr = 0; rr < RPW; rr++) {
            const float Fz = std_zflux<VORD>(b + 1, nz, qfz[rr], wz[rr][1] * tf);
            const float u2 = b + 1 < nz ? half_up(wz[rr][1], dq0[rr], dq1[rr]) : 0.5f * dq0[rr] * wz[rr][1];
            ufzt[rr] = u1lo[rr] + u2;
            mzt[rr] = Fz - ufzt[rr];
        }
        __syncthreads();  // B1
        // beta, cells of tile +1: upwind-only value, in/out sums, bounds, scale factors
        float sic[RPW], soc[RPW];
        {
            const float *QO = PL(C_QO + b % 3);
            const float *U = PL(C_U + b % 3);
            const float *V = PL(C_V + b % 3);
            const float *MX = PL(C_MX), *UX = PL(C_UX), *MY = PL(C_MY), *UY = PL(C_UY);
            float *SI = PL(C_SI), *SO = PL(C_SO);
#pragma unroll
            for (int rr = 0; rr < RPW; rr++) {
                sic[rr] = soc[rr] = 1.0f;
                if (!isE[rr]) continue;
                const int p = pr[rr];
                const float qc = qoz[rr][1], jr = gz[rr][0], djr = dj[rr][1];
                float temp = qc - ((UX[p + 1] - UX[p]) + (UY[p + PW] - UY[p])) / jr;
                temp = temp - (ufzt[rr] - ufzb[rr]) / djr;
                const float xr = MX[p + 1], xl = MX[p], yr_ = MY[p + PW], yl = MY[p], zt = mzt[rr], zb = mzb[rr];
                const float a = -(((fmin_(0.0f, xr) - fmax_(0.0f, xl)) + (fmin_(0.0f, yr_) - fmax_(0.0f, yl))) / jr);
                const float fin = a - (fmin_(0.0f, zt) - fmax_(0.0f, zb)) / djr;
                const float bo = ((fmax_(0.0f, xr) - fmin_(0.0f, xl)) + (fmax_(0.0f, yr_) - fmin_(0.0f, yl))) / jr;
                const float fout = bo + (fmax_(0.0f, zt) - fmin_(0.0f, zb)) / djr;
                float mx = qc, mn = qc;
                if (U[p] > 0.0f) {
                    mx = fmax_(QO[p - 1], mx);
                    mn = fmin_(QO[p - 1], mn);
                } else if (U[p + 1] < 0.0f) {
                    mx = fmax_(QO[p + 1], mx);
                    mn = fmin_(QO[p + 1], mn);
                }
                if (V[p] > 0.0f) {
                    mx = fmax_(QO[p - PW], mx);
                    mn = fmin_(QO[p - PW], mn);
                } else if (V[p + PW] < 0.0f) {
                    mx = fmax_(QO[p + PW], mx);
                    mn = fmin_(QO[p + PW], mn);
                }
                if (b > 0 && wz[rr][0] > 0.0f) {
                    mx = fmax_(qoz[rr][0], mx);
                    mn = fmin_(qoz[rr][0], mn);
                }
                if (b < nz - 1 && wz[rr][1] < 0.0f) {
                    mx = fmax_(qoz[rr][2], mx);
                    mn = fmin_(qoz[rr][2], mn);
                }
                float si = 1.0f, so = 1.0f;
                if (fin > (mx - temp)) si = fmax_(0.0f, (mx - temp) / (fin + e15));
                if (fout > (temp - mn)) so = fmax_(0.0f, (temp - mn) / (fout + e15));
                SI[p] = si;
                SO[p] = so;
                sic[rr] = si;
                soc[rr] = so;
            }
        }
        __syncthreads();  // B2
        // gamma (horizontal update of level b) and delta (vertical update of b-1)
        {
            const float *MX = PL(C_MX), *UX = PL(C_UX), *MY = PL(C_MY), *UY = PL(C_UY);
            const float *SI = PL(C_SI), *SO = PL(C_SO);
#pragma unroll
            for (int rr = 0; rr < RPW; rr++) {
                const int p = pr[rr];
                float tq = 0.0f, fzf = 0.0f;
                if (isT[rr]) {
                    const float fxl = wrf_scaled(MX[p], SI[p], SO[p - 1], SO[p], SI[p - 1]) + UX[p];
                    const float fxr = wrf_scaled(MX[p + 1], SI[p + 1], SO[p], SO[p + 1], SI[p]) + UX[p + 1];
                    const float fyl = wrf_scaled(MY[p], SI[p], SO[p - PW], SO[p], SI[p - PW]) + UY[p];
                    const float fyr = wrf_scaled(MY[p + PW], SI[p + PW], SO[p], SO[p + PW], SI[p]) + UY[p + PW];
                    tq = qoz[rr][1] - ((fxr - fxl) + (fyr - fyl)) / gz[rr][0];
                    const float mz = b >= 1 ? wrf_scaled(mzb[rr], sic[rr], sodn[rr], soc[rr], sidn[rr]) : mzb[rr];
                    fzf = mz + ufzb[rr];
                    if (b >= 1) out[c0[rr] + (size_t)(b - 1) * P] = tqdn[rr] - (fzf - fzfdn[rr]) / dj[rr][0];
                }
                tqdn[rr] = tq;
                fzfdn[rr] = fzf;
                sidn[rr] = sic[rr];
                sodn[rr] = soc[rr];
                ufzb[rr] = ufzt[rr];
                mzb[rr] = mzt[rr];
                dq0[rr] = dq1[rr];
                u1lo[rr] = u1hi[rr];
#pragma unroll
                for (int m = 0; m < 5; m++) qfz[rr][m] = qfz[rr][m + 1];
                qfz[rr][5] = n_qf[rr];
#pragma unroll
                for (int m = 0; m < 3; m++) qoz[rr][m] = qoz[rr][m + 1];
                qoz[rr][3] = n_qo[rr];
                wz[rr][0] = wz[rr][1];
                wz[rr][1] = wz[rr][2];
                wz[rr][2] = n_w[rr];
                gz[rr][0] = gz[rr][1];
                gz[rr][1] = n_g[rr];
                dj[rr][0] = dj[rr][1];
                dj[rr][1] = dj[rr][2];
                dj[rr][2] = n_dj[rr];
            }
        }
    }
    // top face nz is not scaled: (F - uf) + uf
#pragma unroll
    for (int rr = 0; rr < RPW; rr++)
        if (isT[rr]) {
            const float fzf = mzb[rr] + ufzb[rr];
            out[c0[rr] + (size_t)(nz - 1) * P] = tqdn[rr] - (fzf - fzfdn[rr]) / dj[rr][0];
        }
}

// Grid: blockIdx.x = tile * S + species (the species of a tile on
// consecutive CTAs share its Courant and metric planes through L2).
template <int HORD, int VORD, class SH>
__global__ void __launch_bounds__(SH::NT, SH::CORR ? 1 : 3)
    k_std_fused(Geo g, int its, int ite, int jts, int jte, float tf, const __grid_constant__ SpeciesPtrs sp,
                int nspecies, int tiles_x, const float *__restrict__ Um, const float *__restrict__ Vm,
                const float *__restrict__ Wm, const float *__restrict__ Gc, const float *__restrict__ DJR)
{
    extern __shared__ float4 sm4[];
    float *sm = reinterpret_cast<float *>(sm4);
    const int s = blockIdx.x % nspecies;
    const int tile = blockIdx.x / nspecies;
    const int i0 = its + (tile % tiles_x) * SH::TX;
    const int j0 = jts + (tile / tiles_x) * SH::TY;
    if (SH::CORR)
        std_corr_tile<HORD, VORD, SH>(sm, g, its, ite, jts, jte, tf, sp.q1[s], sp.q0[s], sp.out[s], i0, j0, Um, Vm,
                                      Wm, Gc, DJR);
    else
        std_stage_tile<HORD, VORD, SH>(sm, g, its, ite, jts, jte, tf, sp.q1[s], sp.q0[s], sp.out[s], i0, j0, Um,
                                       Vm, Wm, Gc, DJR);
}

using StdStageShape = stdf::Shape<16, 8, false>;
using StdCorrShape = stdf::Shape<28, 32, true>;

template <int HORD, int VORD>
inline cudaError_t std_fused_attr()
{
    cudaError_t e = cudaFuncSetAttribute(k_std_fused<HORD, VORD, StdStageShape>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)stdf::smem_bytes<StdStageShape>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_std_fused<HORD, VORD, StdCorrShape>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)stdf::smem_bytes<StdCorrShape>());
    return e;
}

inline cudaError_t std_fused_setup()
{
    cudaError_t e = cudaSuccess;
#define ICAR_STD_ATTR(h, v) \
    if (e == cudaSuccess) e = std_fused_attr<h, v>();
    ICAR_STD_ATTR(1, 1) ICAR_STD_ATTR(1, 3) ICAR_STD_ATTR(1, 5)
    ICAR_STD_ATTR(3, 1) ICAR_STD_ATTR(3, 3) ICAR_STD_ATTR(3, 5)
    ICAR_STD_ATTR(5, 1) ICAR_STD_ATTR(5, 3) ICAR_STD_ATTR(5, 5)
#undef ICAR_STD_ATTR
    return e;
}

template <int HORD, int VORD, class SH>
inline void std_fused_launch_t(cudaStream_t st, const Geo &g, int hs, float tf, const SpeciesPtrs &sp, int S,
                               const float *Um, const float *Vm, const float *Wm, const float *Gc, const float *DJR)
{
    const int its = hs, ite = g.nx - 1 - hs, jts = hs, jte = g.ny - 1 - hs;
    if (ite < its || jte < jts || S <= 0) return;
    const int tx = (ite - its + SH::TX) / SH::TX, ty = (jte - jts + SH::TY) / SH::TY;
    const unsigned nblk = (unsigned)(tx * ty * S);
    k_std_fused<HORD, VORD, SH><<<nblk, SH::NT, stdf::smem_bytes<SH>(), st>>>(g, its, ite, jts, jte, tf, sp, S, tx,
                                                                              Um, Vm, Wm, Gc, DJR);
}

template <class SH>
inline int std_fused_launch_o(cudaStream_t st, int hord, int vord, const Geo &g, int hs, float tf,
                              const SpeciesPtrs &sp, int S, const float *Um, const float *Vm, const float *Wm,
                              const float *Gc, const float *DJR)
{
#define ICAR_STD_CASE(h, v)                                                         \
    if (hord == h && vord == v) {                                                   \
        std_fused_launch_t<h, v, SH>(st, g, hs, tf, sp, S, Um, Vm, Wm, Gc, DJR);  \
        return 0;                                                                   \
    }
    ICAR_STD_CASE(1, 1) ICAR_STD_CASE(1, 3) ICAR_STD_CASE(1, 5)
    ICAR_STD_CASE(3, 1) ICAR_STD_CASE(3, 3) ICAR_STD_CASE(3, 5)
    ICAR_STD_CASE(5, 1) ICAR_STD_CASE(5, 3) ICAR_STD_CASE(5, 5)
#undef ICAR_STD_CASE
    return 1;
}

// One adv_std_advect3d call for every species: sp.q1 = flux source, sp.q0 =
// qold, sp.out = result (distinct from both).  Returns nonzero for orders
// outside {1,3,5}.
inline int std_fused_launch(cudaStream_t st, bool corr, int hord, int vord, const Geo &g, int hs, float tf,
                            const SpeciesPtrs &sp, int S, const float *Um, const float *Vm, const float *Wm,
                            const float *Gc, const float *DJR)
{
    if (S <= 0) return 0;
    const size_t ring = ((size_t)g.nx * 2 * hs + (size_t)2 * hs * (size_t)(g.ny > 2 * hs ? g.ny - 2 * hs : 0)) *
                        (size_t)g.nz * (size_t)S;
    if (ring > 0) {
        const unsigned nb = (unsigned)std::min<size_t>((ring + 255) / 256, 148 * 8);
        k_std_ring<<<nb, 256, 0, st>>>(g, hs, sp, S);
    }
    return corr ? std_fused_launch_o<StdCorrShape>(st, hord, vord, g, hs, tf, sp, S, Um, Vm, Wm, Gc, DJR)
                : std_fused_launch_o<StdStageShape>(st, hord, vord, g, hs, tf, sp, S, Um, Vm, Wm, Gc, DJR);
}

}  // namespace icar
