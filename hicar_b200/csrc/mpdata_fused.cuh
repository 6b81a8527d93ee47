// Fused MPDATA step for the configuration ICAR runs (mpdata_order 2, with or
// without the FCT limiter).  Two kernels per step:
//
//   k_mp_prep     species-independent per-step fields: the Courant fluxes
//                 U_m, V_m, W_m (mpdata_compute_wind) plus G = J*rho,
//                 DJR = dz*J*rho and W' = W_m/dz, formed with exactly the
//                 reference's operations so every later use is bit-identical.
//   k_mp_upwind_cols  donor-cell pass q0 -> q1 (upwind_advection,
//                 adv_mpdata.f90:43-103), one thread per column marching up
//                 it over staged level planes; also writes the untouched
//                 boundary ring of the output.
//   k_mp_corr     antidiffusive pseudo-velocities, FCT limiter and the
//                 corrective donor-cell pass, fused: one CTA owns a 28x16
//                 column tile of one species and marches up the column,
//                 keeping rolling z-windows of q0/q1/winds in shared memory
//                 and the per-column z-state in registers, so every
//                 intermediate of the reference (u2/v2/w2, the limiter's
//                 bounds and fluxes) stays on chip.
//
// Reference: src/physics/adv_mpdata.f90:43-413, adv_mpdata_FCT_core.f90:47-116.
// The limiter is applied in its per-cell form (see fct_cell_terms in
// mpdata_kernels.cuh): each cell's in/out bounds and flux sums are computed
// once per direction and every face reads the two cells beside it.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace icar {

// --------------------------------------------------------------------------
// per-step species-independent fields
// --------------------------------------------------------------------------
__global__ void k_mp_prep(Geo g, float dx, float dt, int adv_den, const float *__restrict__ u,
                          const float *__restrict__ v, const float *__restrict__ w, const float *__restrict__ rho,
                          const float *__restrict__ jac, const float *__restrict__ ju, const float *__restrict__ jv,
                          const float *__restrict__ jw, const float *__restrict__ dz, float *__restrict__ Um,
                          float *__restrict__ Vm, float *__restrict__ Wm, float *__restrict__ Gc,
                          float *__restrict__ DJR, float *__restrict__ Wp)
{
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int ni = g.nx + 1, nk = g.nz, nj = g.ny + 1;
    const int i = (int)(t % (size_t)ni);
    size_t rest = t / (size_t)ni;
    const int k = (int)(rest % (size_t)nk);
    const int j = (int)(rest / (size_t)nk);
    if (j >= nj) return;
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
            float wm;
            if (k < g.nz - 1) {
                float r1 = adv_den ? rho[ix(g, i, k + 1, j)] : 1.0f;
                wm = w[c] * dt * jw[c] * (r1 + r0) * 0.5f;
            } else {
                wm = w[c] * dt * jw[c] * r0;
            }
            Wm[c] = wm;
            const float d = dz[c], jj = jac[c], rh = rho[c];
            Gc[c] = jj * rh;
            DJR[c] = d * jj * rh;
            Wp[c] = wm / d;
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

// Species pointer tables for the multi-species launches.
struct SpeciesPtrs {
    const float *q0[32];
    float *q1[32];
    float *out[32];
};

// Species per group of the donor-cell pass for the knob sg (0 = all species).
__host__ __device__ inline int upwind_group(int S, int sg) { return sg <= 0 || sg > S ? S : sg; }

namespace mpf {
constexpr int TX = 28;            // output columns per tile
constexpr int PW = 32;            // plane width: x from i0-2 to i0+29
// Tile heights: TY output rows, NW warps, TY/NW output rows per warp; the
// plane holds TY+4 rows (y from j0-2 to j0+TY+1).
template <int TY_, int NW_>
struct Shape {
    static constexpr int TY = TY_;
    static constexpr int NW = NW_;
    static constexpr int NT = 32 * NW_;
    static constexpr int PH = TY_ + 4;
    static constexpr int PLANE = PW * PH;
    static constexpr int RPW = (TY_ + NW_ - 1) / NW_;
    // one warp beyond the output rows (NW = TY+1): it owns no output row and
    // takes the face and limiter rows a tile has beyond TY, so every warp
    // does the same number of rows per level
    static constexpr bool EXTRA = NW_ == TY_ + 1;
    static_assert(TY_ % NW_ == 0 || EXTRA, "rows per warp must be whole");
};
// shared-memory plane slots
constexpr int S_Q1 = 0;           // 4 ring slots: level l -> S_Q1 + (l & 3)
constexpr int S_Q0 = 4;           // 3 ring slots: level l -> S_Q0 + l % 3
constexpr int S_U = 7;            // U_m, 3 slots
constexpr int S_V = 10;           // V_m, 3 slots
constexpr int S_W = 13;           // W' = W_m/dz, 3 slots
constexpr int S_G = 16;           // G = J*rho, 3 slots
constexpr int S_U2 = 19, S_V2 = 20;  // unlimited pseudo-velocities of level t
constexpr int S_BXI = 21, S_BXO = 22, S_BYI = 23, S_BYO = 24;
constexpr int NPLANES = 25;
template <class SH>
constexpr size_t smem_bytes() { return (size_t)NPLANES * SH::PLANE * sizeof(float); }
}  // namespace mpf

__device__ __forceinline__ void cp_async16(float *dst, const float *src, bool valid)
{
    unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Donor-cell pass 1 for every species of a species group, one thread per
// column marching up the column (the donor-cell arithmetic of upwind_advection, cell
// for cell).  CTA tile 32 x 8 columns; blockIdx.z selects the species
// group.  Each level of every species of the group, and of U_m and V_m,
// arrives in shared-memory planes by 16-byte cp.async three levels ahead
// (planes span x from i0-4 to i0+35 and y from j0-1 to j0+8, covering the
// stencil's x/y neighbours); the vertical neighbours come from the planes
// of the levels above and below, W_m, G and DJR from the column itself.
// Boundary-ring columns copy q0 to the pass-1 and output buffers.
namespace upf {
constexpr int BX = 32, BY = 8, NT = BX * BY;
constexpr int PW = 40, PH = BY + 2, PLANE = PW * PH, CPR = PW / 4;
constexpr int SGMAX = 6;                 // species per CTA
constexpr int NSL = 5;                   // level slots: k-1 .. k+3
constexpr int NPL = SGMAX + 2;           // species planes, then U_m, V_m
constexpr int NCH = (NPL * CPR * PH + NT - 1) / NT;
constexpr size_t SMEM = (size_t)NSL * NPL * PLANE * sizeof(float);
}  // namespace upf

// One 32 x 8 column tile (first column i0, first row j0) for species
// q0s[0..n), n <= upf::SGMAX; sm is the CTA's dynamic shared memory.
__device__ __forceinline__ void upwind_cols_tile(float *sm, const Geo &g, const float *const *q0s, float *const *q1s,
                                                 float *const *outs, int n, int i0, int j0,
                                                 const float *__restrict__ U, const float *__restrict__ V,
                                                 const float *__restrict__ W, const float *__restrict__ Gc,
                                                 const float *__restrict__ DJR)
{
    using namespace upf;
    const int tx = threadIdx.x % BX, ty = threadIdx.x / BX;
    const int i = i0 + tx, j = j0 + ty;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int ox = i0 - 4, oy = j0 - 1;
    const bool in = i < nx && j < ny;
    const bool ring = i == 0 || i == nx - 1 || j == 0 || j == ny - 1;
    // this thread's chunks of one level: plane p (species 0..n-1, U, V), row, chunk
    const float *src[NCH];
    size_t off[NCH];
    int dst[NCH];
    bool ok[NCH];
#pragma unroll
    for (int c = 0; c < NCH; c++) {
        const int e = threadIdx.x + c * NT;
        dst[c] = -1;
        ok[c] = false;
        off[c] = 0;
        src[c] = U;
        if (e < NPL * CPR * PH) {
            const int p = e / (CPR * PH), r = e % (CPR * PH);
            const int ly = r / CPR, cx = r % CPR;
            const bool use = p < n || p >= SGMAX;
            if (use) {
                const int gi = ox + 4 * cx, gj = oy + ly;
                const bool yface = p == SGMAX + 1;
                dst[c] = p * PLANE + ly * PW + 4 * cx;
                src[c] = p < SGMAX ? q0s[p] : (yface ? V : U);
                ok[c] = gi >= 0 && gi < g.P && gj >= 0 && gj < (yface ? ny + 1 : ny);
                if (ok[c]) off[c] = (size_t)gi + (size_t)g.P * nz * gj;
            }
        }
    }
    auto issue = [&](int k) {
        if (k < nz) {
            float *slot = sm + (size_t)(k % NSL) * NPL * PLANE;
            const size_t lo = (size_t)k * g.P;
#pragma unroll
            for (int c = 0; c < NCH; c++)
                if (dst[c] >= 0) cp_async16(slot + dst[c], ok[c] ? src[c] + off[c] + lo : src[c], ok[c]);
        }
        cp_async_commit();
    };
    issue(0);
    issue(1);
    issue(2);
    const int pc = (j - oy) * PW + (i - ox);
    const size_t c0 = in ? ix(g, i, 0, j) : 0, sz = (size_t)g.P;
    float wb = 0.0f;  // W_m one level down
    float n_wt = in ? W[c0] : 0.0f, n_G = in ? Gc[c0] : 0.0f, n_djr = in ? DJR[c0] : 0.0f;
    for (int k = 0; k < nz; k++) {
        cp_async_wait<1>();   // levels up to k+1 have landed
        __syncthreads();      // and every thread is done with level k-1
        issue(k + 3);         // into the slot of level k-2
        const float wt = n_wt, G = n_G, djr = n_djr;
        if (in && k + 1 < nz) {
            n_wt = W[c0 + (k + 1) * sz];
            n_G = Gc[c0 + (k + 1) * sz];
            n_djr = DJR[c0 + (k + 1) * sz];
        }
        if (!in) continue;
        const float *L = sm + (size_t)(k % NSL) * NPL * PLANE;
        const float *Lu = sm + (size_t)((k + 1) % NSL) * NPL * PLANE;
        const float *Ld = sm + (size_t)((k + NSL - 1) % NSL) * NPL * PLANE;
        const size_t c = c0 + k * sz;
        if (ring) {
            for (int u = 0; u < n; u++) {
                const float q0 = L[u * PLANE + pc];
                q1s[u][c] = q0;
                outs[u][c] = q0;
            }
        } else {
            const float ue = L[SGMAX * PLANE + pc + 1], uw = L[SGMAX * PLANE + pc];
            const float vn = L[(SGMAX + 1) * PLANE + pc + PW], vs = L[(SGMAX + 1) * PLANE + pc];
            const bool mid = k > 0 && k < nz - 1;
            for (int u = 0; u < n; u++) {
                const float *Q = L + u * PLANE + pc;
                const float q0 = Q[0];
                const float fe = flux1(q0, Q[1], ue);
                const float fw = flux1(Q[-1], q0, uw);
                const float f3 = flux1(q0, Q[PW], vn);
                const float f4 = flux1(Q[-PW], q0, vs);
                float val = q0 - ((fe - fw) + (f3 - f4)) / G;
                if (mid) {
                    const float f5t = flux1(q0, Lu[u * PLANE + pc], wt);
                    const float f5b = flux1(Ld[u * PLANE + pc], q0, wb);
                    val = val - (f5t - f5b) / djr;
                } else if (k == 0) {
                    const float f5t = flux1(q0, Lu[u * PLANE + pc], wt);
                    val = val - f5t / djr;
                } else {
                    const float f5b = flux1(Ld[u * PLANE + pc], q0, wb);
                    val = val - (q0 * wt - f5b) / djr;
                }
                q1s[u][c] = val;
            }
        }
        wb = wt;
    }
    cp_async_wait<0>();
}

__global__ void __launch_bounds__(upf::NT)
    k_mp_upwind_cols(Geo g, const __grid_constant__ SpeciesPtrs sp, int S, int sg, const float *__restrict__ U,
                     const float *__restrict__ V, const float *__restrict__ W, const float *__restrict__ Gc,
                     const float *__restrict__ DJR)
{
    extern __shared__ float4 sm4[];
    const int s0 = blockIdx.z * sg;
    upwind_cols_tile(reinterpret_cast<float *>(sm4), g, sp.q0 + s0, sp.q1 + s0, sp.out + s0, min(sg, S - s0),
                     blockIdx.x * upf::BX, blockIdx.y * upf::BY, U, V, W, Gc, DJR);
}


// Beta of the FCT limiter, num/den with den > 0 and num >= 0.  Only
// min(1, beta) is ever used, so a quotient >= 1 is returned as 1 without
// dividing (num >= den implies RN(num/den) >= 1), and num == 0 gives +0
// exactly as the division would; every other case divides.
__device__ __forceinline__ float fct_beta(float num, float den)
{
    if (num >= den) return 1.0f;
    if (num == 0.0f) return 0.0f;
    return num / den;
}

// Asynchronous copies of one level of a 3-D field into a plane slot, in
// 16-byte chunks.  The plane starts at x = i0-2, a multiple of 4, so every
// chunk is either wholly inside a row's pitch (valid cells, or the zero
// padding past nx) or wholly outside the field and zero-filled.  Chunk
// e = tid + c*NT covers x from i0-2+4*(e%8) in row j0-2+e/8; its source
// offset at level 0 and whether it lies inside a cell field (rows < ny) or
// a y-face field (rows <= ny) are fixed for the whole tile, so copying a
// level costs one add and one cp.async per chunk.
template <class SH>
struct PlaneLoader {
    static constexpr int NCH = ((mpf::PW / 4) * SH::PH + SH::NT - 1) / SH::NT;
    size_t off[NCH];
    int dst[NCH];
    unsigned okc, okv;
    size_t lstride;
    __device__ __forceinline__ PlaneLoader(const Geo &g, int i0, int j0) : okc(0u), okv(0u), lstride((size_t)g.P)
    {
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            const int e = threadIdx.x + c * SH::NT;
            dst[c] = -1;
            off[c] = 0;
            if (e < (mpf::PW / 4) * SH::PH) {
                const int cx = e % (mpf::PW / 4), ly = e / (mpf::PW / 4);
                const int i = i0 - 2 + 4 * cx, j = j0 - 2 + ly;
                dst[c] = ly * mpf::PW + 4 * cx;
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

// IEEE-rounded quotient (a zero-numerator shortcut was measured slower: the
// branch costs more than the divisions it skips in mixed warps).
__device__ __forceinline__ float div0(float n, float d) { return n / d; }

// Limited pseudo-velocity at a face (flux_limiter, adv_mpdata_FCT_core.f90):
// flow towards +x/+y/+z takes beta_in of the cell after the face and
// beta_out of the cell before it, flow the other way the opposite pair.
__device__ __forceinline__ float fct_limit(float u, float bin_r, float bout_l, float bin_l, float bout_r)
{
    if (u > 0.0f) return fminf(fminf(1.0f, bin_r), bout_l) * u;
    if (u < 0.0f) return fminf(fminf(1.0f, bin_l), bout_r) * u;
    return u;
}

// One 28 x TY column tile of one species: the z-march described at the top
// of this file.  i0 is the first output column (i0-2 a multiple of 4), j0
// the first output row; sm is the CTA's dynamic shared memory.
template <bool FCT, class SH>
__device__ __forceinline__ void mp_corr_tile(float *sm, const Geo &g, const float *__restrict__ q0g,
                                             const float *__restrict__ q1g, float *__restrict__ outg, int i0, int j0,
                                             const float *__restrict__ Um, const float *__restrict__ Vm,
                                             const float *__restrict__ Wp, const float *__restrict__ Gc,
                                             const float *__restrict__ DJR, const float *__restrict__ dz)
{
    using namespace mpf;
    constexpr int TY = SH::TY, NW = SH::NW, PH = SH::PH, PLANE = SH::PLANE, RPW = SH::RPW;
    (void)PH;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int lane = threadIdx.x & 31, warp = __shfl_sync(0xffffffffu, (int)(threadIdx.x >> 5), 0);
    const float e10 = 1e-10f, e15 = 1e-15f, q4 = 1.0f / 4.0f;
    auto P = [&](int slot) { return sm + (size_t)slot * PLANE; };
#define AT(slot, lx, ly) sm[(size_t)(slot) * PLANE + (ly) * PW + (lx)]

    const PlaneLoader<SH> pl(g, i0, j0);
    // ---- prologue: levels 0 and 1 of everything the first iteration reads
    pl.load(P(S_Q1 + 0), q1g, 0, false);
    pl.load(P(S_Q0 + 0), q0g, 0, false);
    pl.load(P(S_U + 0), Um, 0, false);
    pl.load(P(S_V + 0), Vm, 0, true);
    pl.load(P(S_W + 0), Wp, 0, false);
    pl.load(P(S_G + 0), Gc, 0, false);
    pl.load(P(S_Q1 + 1), q1g, 1, false);
    pl.load(P(S_Q0 + 1), q0g, 1, false);
    pl.load(P(S_U + 1), Um, 1, false);
    pl.load(P(S_V + 1), Vm, 1, true);
    pl.load(P(S_G + 1), Gc, 1, false);
    cp_async_commit();

    // per-output-cell z state (RPW output rows per warp)
    // r_q1dn / r_q0dn: q1 and q0 one level below the level being limited;
    // r_q1dd: q1 two levels below (the level under the corrective pass).
    float r_fz[RPW], r_w2[RPW], r_bzi[RPW], r_bzo[RPW], r_w2l[RPW], r_q1dn[RPW], r_q0dn[RPW], r_q1dd[RPW];
    // r_part: the horizontal part of the corrective pass one level below.
    float r_part[RPW], r_DJR[RPW];
#pragma unroll
    for (int rr = 0; rr < RPW; rr++) {
        r_fz[rr] = r_w2[rr] = r_bzi[rr] = r_bzo[rr] = r_w2l[rr] = r_q1dn[rr] = r_q0dn[rr] = r_q1dd[rr] = 0.0f;
        r_part[rr] = 0.0f;
        r_DJR[rr] = 1.0f;
    }

    for (int t = 0; t <= nz; t++) {
        // planes of level t+1 (and W' of level t) must have landed
        cp_async_wait<0>();
        __syncthreads();
        // prefetch the levels the next iteration adds: q1/q0/U/V/G at t+2, W' at t+1
        if (t + 2 < nz) {
            pl.load(P(S_Q1 + ((t + 2) & 3)), q1g, t + 2, false);
            pl.load(P(S_Q0 + (t + 2) % 3), q0g, t + 2, false);
            pl.load(P(S_U + (t + 2) % 3), Um, t + 2, false);
            pl.load(P(S_V + (t + 2) % 3), Vm, t + 2, true);
            pl.load(P(S_G + (t + 2) % 3), Gc, t + 2, false);
        }
        if (t + 1 < nz) pl.load(P(S_W + (t + 1) % 3), Wp, t + 1, false);
        cp_async_commit();

        const bool haveA = t < nz;
        const int sQm = S_Q1 + ((t + 3) & 3), sQc = S_Q1 + (t & 3), sQp = S_Q1 + ((t + 1) & 3);
        const int sQ0c = S_Q0 + t % 3, sQ0p = S_Q0 + (t + 1) % 3;
        const int sUc = S_U + t % 3, sUp = S_U + (t + 1) % 3;
        const int sVc = S_V + t % 3, sVp = S_V + (t + 1) % 3;
        const int sWc = S_W + t % 3, sWm = S_W + (t + 2) % 3;
        const int sGc = S_G + t % 3, sGp = S_G + (t + 1) % 3;
        const bool kint = t > 0 && t < nz - 1;

        float n_fz[RPW], n_w2[RPW], n_bzi[RPW] = {}, n_bzo[RPW] = {}, n_w2l[RPW], n_part[RPW];
        if (haveA) {
            // ---------------- A1: u2, v2 at level t; w2 at the top of t --------
            for (int r = warp; r < TY; r += NW) {  // u2 faces x in [-1, TX+1] -> lx 1..31
                const int ly = r + 2, lx = lane;
                const int f = i0 - 2 + lx, j = j0 - 2 + ly;
                float u2 = 0.0f;
                if (lx >= 1 && f >= 1 && f <= nx - 1 && j <= ny - 1) {
                    const float rx = AT(sQc, lx, ly), lq = AT(sQc, lx - 1, ly);
                    const float uu = AT(sUc, lx, ly);
                    const float Gs = AT(sGc, lx, ly) + AT(sGc, lx - 1, ly);
                    const float denom = rx + lq + e10;
                    float val = fabsf(uu) * (1.0f - fabsf(uu) / (0.5f * Gs));
                    val = div0(val * (rx - lq), denom);
                    if (j > 0 && j < ny - 1) {
                        const float a = AT(sQc, lx, ly + 1), b = AT(sQc, lx, ly - 1);
                        const float c = AT(sQc, lx - 1, ly + 1), d = AT(sQc, lx - 1, ly - 1);
                        const float eq = div0(a - b + c - d, a + b + c + d + e10);
                        const float ev = q4 * (AT(sVc, lx, ly) + AT(sVc, lx, ly + 1) + AT(sVc, lx - 1, ly) +
                                               AT(sVc, lx - 1, ly + 1));
                        val = val - div0(0.5f * uu * ev * eq, Gs);
                    }
                    if (kint) {
                        const float a = AT(sQp, lx, ly), b = AT(sQm, lx, ly);
                        const float c = AT(sQp, lx - 1, ly), d = AT(sQm, lx - 1, ly);
                        const float eq = div0(a - b + c - d, a + b + c + d + e10);
                        const float ev = q4 * (AT(sWc, lx, ly) + AT(sWm, lx, ly) + AT(sWc, lx - 1, ly) +
                                               AT(sWm, lx - 1, ly));
                        val = val - div0(0.5f * uu * ev * eq, Gs);
                    }
                    u2 = val * 0.5f;
                }
                AT(S_U2, lx, ly) = u2;
            }
            for (int r = SH::EXTRA && warp == TY ? TY : warp; r < (!SH::EXTRA ? TY + 3 : warp == TY ? TY + 3 : warp + 1);
                 r += SH::EXTRA ? 1 : NW) {  // v2 faces y in [-1, TY+1] -> ly 1..TY+3
                const int ly = r + 1, lx = lane;
                const int i = i0 - 2 + lx, gf = j0 - 2 + ly;
                float v2 = 0.0f;
                if (lx >= 2 && lx < TX + 2 && i >= 0 && i <= nx - 1 && gf >= 1 && gf <= ny - 1) {
                    const float rq = AT(sQc, lx, ly), lq = AT(sQc, lx, ly - 1);
                    const float vv = AT(sVc, lx, ly);
                    const float Gs = AT(sGc, lx, ly) + AT(sGc, lx, ly - 1);
                    const float denom = rq + lq + e10;
                    float val = fabsf(vv) * (1.0f - fabsf(vv) / (0.5f * Gs));
                    val = div0(val * (rq - lq), denom);
                    float ev = 0.0f, eq = 0.0f;
                    if (i > 0 && i < nx - 1) {
                        const float A = AT(sQc, lx + 1, ly - 1), B = AT(sQc, lx - 1, ly);
                        const float C = AT(sQc, lx + 1, ly), D = AT(sQc, lx - 1, ly - 1);
                        eq = div0(A - B + C - D, C + A + B + D + e10);
                        ev = q4 * (AT(sUc, lx + 1, ly) + AT(sUc, lx + 1, ly - 1) + AT(sUc, lx, ly) +
                                   AT(sUc, lx, ly - 1));
                    }
                    val = val - div0(0.5f * vv * ev * eq, Gs);
                    if (kint) {
                        const float A = AT(sQp, lx, ly - 1), B = AT(sQm, lx, ly);
                        const float C = AT(sQp, lx, ly), D = AT(sQm, lx, ly - 1);
                        const float eq2 = div0(A - B + C - D, A + B + C + D + e10);
                        const float ev2 = q4 * (AT(sWc, lx, ly) + AT(sWm, lx, ly) + AT(sWc, lx, ly - 1) +
                                                AT(sWm, lx, ly - 1));
                        val = val - div0(0.5f * vv * ev2 * eq2, Gs);
                    }
                    v2 = val * 0.5f;
                }
                AT(S_V2, lx, ly) = v2;
            }
#pragma unroll
            for (int rr = 0; rr < RPW; rr++) {  // w2 at the top face of level t, output cells
                const int ly = warp + NW * rr + 2, lx = lane + 2;
                float w2 = 0.0f, fz = 0.0f;
                const int iw = i0 - 2 + lx, jw = j0 - 2 + ly;
                if (warp + NW * rr < TY && lane < TX && t < nz - 1 && iw >= 1 && iw <= nx - 2 && jw <= ny - 2) {
                    const float rq = AT(sQp, lx, ly), lq = AT(sQc, lx, ly);
                    const float ww = AT(sWc, lx, ly);
                    const float Gs = AT(sGp, lx, ly) + AT(sGc, lx, ly);
                    const float denom = rq + lq + e10;
                    float val = fabsf(ww) * (1.0f - fabsf(ww) / (0.5f * Gs));
                    val = div0(val * (rq - lq), denom);
                    {
                        const float A = AT(sQp, lx + 1, ly), B = AT(sQc, lx - 1, ly);
                        const float C = AT(sQc, lx + 1, ly), D = AT(sQp, lx - 1, ly);
                        const float eq = div0(A - B + C - D, C + A + B + D + e10);
                        const float ev = q4 * (AT(sUc, lx + 1, ly) + AT(sUp, lx + 1, ly) + AT(sUc, lx, ly) +
                                               AT(sUp, lx, ly));
                        val = val - div0(0.5f * ww * ev * eq, Gs);
                    }
                    {
                        const float A = AT(sQp, lx, ly + 1), B = AT(sQc, lx, ly - 1);
                        const float C = AT(sQc, lx, ly + 1), D = AT(sQp, lx, ly - 1);
                        const float eq2 = div0(A - B + C - D, C + D + A + B + e10);
                        const float ev2 = q4 * (AT(sVc, lx, ly) + AT(sVp, lx, ly) + AT(sVc, lx, ly + 1) +
                                                AT(sVp, lx, ly + 1));
                        val = val - div0(0.5f * ww * ev2 * eq2, Gs);
                    }
                    w2 = val * 0.5f * dz[ix(g, iw, t, jw)];
                    fz = flux1(lq, rq, w2);
                }
                n_w2[rr] = w2;
                n_fz[rr] = fz;
            }
            __syncthreads();

            if (FCT) {
                // ------------- A2: per-cell limiter terms at level t ---------
                for (int r = warp; r < TY; r += NW) {  // x: cells x in [-1, TX] -> lx 1..TX+2
                    const int ly = r + 2, lx = lane;
                    const int i = i0 - 2 + lx;
                    if (lx >= 1 && lx <= TX + 2 && i >= 0 && i <= nx - 1) {
                        float qmax, qmin, fin, fout;
                        const float qc = AT(sQc, lx, ly);
                        if (i == 0) {
                            qmax = fmaxf(fmaxf(qc, AT(sQc, lx + 1, ly)), fmaxf(AT(sQ0c, lx, ly), AT(sQ0c, lx + 1, ly)));
                            qmin = fminf(fminf(qc, AT(sQc, lx + 1, ly)), fminf(AT(sQ0c, lx, ly), AT(sQ0c, lx + 1, ly)));
                            fin = 0.0f;
                            fout = 0.0f;
                        } else if (i == nx - 1) {
                            qmax = fmaxf(fmaxf(AT(sQc, lx - 1, ly), qc), AT(sQ0c, lx - 1, ly));
                            qmin = fminf(fminf(AT(sQc, lx - 1, ly), qc), AT(sQ0c, lx - 1, ly));
                            fin = 0.0f;
                            fout = 0.0f;
                        } else {
                            qmax = fmaxf(fmaxf(fmaxf(AT(sQc, lx - 1, ly), qc), AT(sQc, lx + 1, ly)),
                                         fmaxf(fmaxf(AT(sQ0c, lx - 1, ly), AT(sQ0c, lx, ly)), AT(sQ0c, lx + 1, ly)));
                            qmin = fminf(fminf(fminf(AT(sQc, lx - 1, ly), qc), AT(sQc, lx + 1, ly)),
                                         fminf(fminf(AT(sQ0c, lx - 1, ly), AT(sQ0c, lx, ly)), AT(sQ0c, lx + 1, ly)));
                            const float fl = flux1(AT(sQc, lx - 1, ly), qc, AT(S_U2, lx, ly));
                            const float fr = flux1(qc, AT(sQc, lx + 1, ly), AT(S_U2, lx + 1, ly));
                            fin = fmaxf(0.0f, fl) - fminf(0.0f, fr);
                            fout = fmaxf(0.0f, fr) - fminf(0.0f, fl);
                        }
                        AT(S_BXI, lx, ly) = fct_beta(qmax - qc, fin + e15);
                        AT(S_BXO, lx, ly) = fct_beta(qc - qmin, fout + e15);
                    }
                }
                for (int r = SH::EXTRA && warp == TY ? TY : warp;
                     r < (!SH::EXTRA ? TY + 2 : warp == TY ? TY + 2 : warp + 1);
                     r += SH::EXTRA ? 1 : NW) {  // y: cells y in [-1, TY] -> ly 1..TY+2
                    const int ly = r + 1, lx = lane;
                    const int j = j0 - 2 + ly;
                    if (lx >= 2 && lx < TX + 2 && j <= ny - 1) {
                        float qmax, qmin, fin, fout;
                        const float qc = AT(sQc, lx, ly);
                        if (j == 0) {
                            qmax = fmaxf(fmaxf(qc, AT(sQc, lx, ly + 1)), fmaxf(AT(sQ0c, lx, ly), AT(sQ0c, lx, ly + 1)));
                            qmin = fminf(fminf(qc, AT(sQc, lx, ly + 1)), fminf(AT(sQ0c, lx, ly), AT(sQ0c, lx, ly + 1)));
                            fin = 0.0f;
                            fout = 0.0f;
                        } else if (j == ny - 1) {
                            qmax = fmaxf(fmaxf(AT(sQc, lx, ly - 1), qc), AT(sQ0c, lx, ly - 1));
                            qmin = fminf(fminf(AT(sQc, lx, ly - 1), qc), AT(sQ0c, lx, ly - 1));
                            fin = 0.0f;
                            fout = 0.0f;
                        } else {
                            qmax = fmaxf(fmaxf(fmaxf(AT(sQc, lx, ly - 1), qc), AT(sQc, lx, ly + 1)),
                                         fmaxf(fmaxf(AT(sQ0c, lx, ly - 1), AT(sQ0c, lx, ly)), AT(sQ0c, lx, ly + 1)));
                            qmin = fminf(fminf(fminf(AT(sQc, lx, ly - 1), qc), AT(sQc, lx, ly + 1)),
                                         fminf(fminf(AT(sQ0c, lx, ly - 1), AT(sQ0c, lx, ly)), AT(sQ0c, lx, ly + 1)));
                            const float fl = flux1(AT(sQc, lx, ly - 1), qc, AT(S_V2, lx, ly));
                            const float fr = flux1(qc, AT(sQc, lx, ly + 1), AT(S_V2, lx, ly + 1));
                            fin = fmaxf(0.0f, fl) - fminf(0.0f, fr);
                            fout = fmaxf(0.0f, fr) - fminf(0.0f, fl);
                        }
                        AT(S_BYI, lx, ly) = fct_beta(qmax - qc, fin + e15);
                        AT(S_BYO, lx, ly) = fct_beta(qc - qmin, fout + e15);
                    }
                }
#pragma unroll
                for (int rr = 0; rr < RPW; rr++) {  // z: the output cell at level t
                    const int ly = warp + NW * rr + 2, lx = lane + 2;
                    float bzi = 0.0f, bzo = 0.0f;
                    if (warp + NW * rr < TY && lane < TX) {
                        float qmax, qmin, fin, fout;
                        const float qc = AT(sQc, lx, ly), q0c = AT(sQ0c, lx, ly);
                        if (t == 0) {
                            const float qu = AT(sQp, lx, ly), q0u = AT(sQ0p, lx, ly);
                            qmax = fmaxf(fmaxf(qc, qu), fmaxf(q0c, q0u));
                            qmin = fminf(fminf(qc, qu), fminf(q0c, q0u));
                            fin = 0.0f - fminf(0.0f, n_fz[rr]);
                            fout = fmaxf(0.0f, n_fz[rr]);
                        } else if (t == nz - 1) {
                            qmax = fmaxf(fmaxf(r_q1dn[rr], qc), r_q0dn[rr]);
                            qmin = fminf(fminf(r_q1dn[rr], qc), r_q0dn[rr]);
                            fin = fmaxf(0.0f, r_fz[rr]) - fminf(0.0f, r_fz[rr]);
                            fout = fin;
                        } else {
                            const float qu = AT(sQp, lx, ly), q0u = AT(sQ0p, lx, ly);
                            qmax = fmaxf(fmaxf(fmaxf(r_q1dn[rr], qc), qu), fmaxf(fmaxf(r_q0dn[rr], q0c), q0u));
                            qmin = fminf(fminf(fminf(r_q1dn[rr], qc), qu), fminf(fminf(r_q0dn[rr], q0c), q0u));
                            fin = fmaxf(0.0f, r_fz[rr]) - fminf(0.0f, n_fz[rr]);
                            fout = fmaxf(0.0f, n_fz[rr]) - fminf(0.0f, r_fz[rr]);
                        }
                        bzi = fct_beta(qmax - qc, fin + e15);
                        bzo = fct_beta(qc - qmin, fout + e15);
                    }
                    n_bzi[rr] = bzi;
                    n_bzo[rr] = bzo;
                }
                __syncthreads();
            }
            // ------- B1: horizontal part of the corrective pass at level t --------
            // The limited face velocities are formed here from the unlimited
            // ones and the limiter terms of the two cells beside each face;
            // the result waits in a register for the vertical part (B2).
#pragma unroll
            for (int rr = 0; rr < RPW; rr++) {
                const int ly = warp + NW * rr + 2, lx = lane + 2;
                const int i = i0 - 2 + lx, j = j0 - 2 + ly;
                n_part[rr] = 0.0f;
                if (warp + NW * rr < TY && lane < TX && i >= 1 && i <= nx - 2 && j <= ny - 2) {
                    float uw = AT(S_U2, lx, ly), ue = AT(S_U2, lx + 1, ly);
                    float vs = AT(S_V2, lx, ly), vn = AT(S_V2, lx, ly + 1);
                    if (FCT) {
                        const float bxi_c = AT(S_BXI, lx, ly), bxo_c = AT(S_BXO, lx, ly);
                        const float byi_c = AT(S_BYI, lx, ly), byo_c = AT(S_BYO, lx, ly);
                        uw = fct_limit(uw, bxi_c, AT(S_BXO, lx - 1, ly), AT(S_BXI, lx - 1, ly), bxo_c);
                        ue = fct_limit(ue, AT(S_BXI, lx + 1, ly), bxo_c, bxi_c, AT(S_BXO, lx + 1, ly));
                        vs = fct_limit(vs, byi_c, AT(S_BYO, lx, ly - 1), AT(S_BYI, lx, ly - 1), byo_c);
                        vn = fct_limit(vn, AT(S_BYI, lx, ly + 1), byo_c, byi_c, AT(S_BYO, lx, ly + 1));
                    }
                    const float qc = AT(sQc, lx, ly);
                    const float fe = flux1(qc, AT(sQc, lx + 1, ly), ue);
                    const float fw = flux1(AT(sQc, lx - 1, ly), qc, uw);
                    const float f3 = flux1(qc, AT(sQc, lx, ly + 1), vn);
                    const float f4 = flux1(AT(sQc, lx, ly - 1), qc, vs);
                    n_part[rr] = qc - div0((fe - fw) + (f3 - f4), AT(sGc, lx, ly));
                }
                // limited w2 at the top face of level t-1
                float w = r_w2[rr];
                if (FCT && t >= 1) w = fct_limit(w, n_bzi[rr], r_bzo[rr], r_bzi[rr], n_bzo[rr]);
                n_w2l[rr] = w;
            }
        } else {
#pragma unroll
            for (int rr = 0; rr < RPW; rr++) {
                n_w2l[rr] = 0.0f;  // top face of the model: w2(kme) = 0
                n_fz[rr] = n_w2[rr] = n_bzi[rr] = n_bzo[rr] = n_part[rr] = 0.0f;
            }
        }

        // ---------------- B2: finish the corrective pass at level t-1 ----------
        if (t >= 1) {
            const int L = t - 1;
#pragma unroll
            for (int rr = 0; rr < RPW; rr++) {
                const int ly = warp + NW * rr + 2, lx = lane + 2;
                const int i = i0 - 2 + lx, j = j0 - 2 + ly;
                if (warp + NW * rr < TY && lane < TX && i >= 1 && i <= nx - 2 && j <= ny - 2) {
                    const float qc = r_q1dn[rr];
                    const float wtop = n_w2l[rr], wbot = r_w2l[rr];
                    float val = r_part[rr];
                    if (L > 0 && L < nz - 1) {
                        const float f5t = flux1(qc, AT(sQc, lx, ly), wtop);
                        const float f5b = flux1(r_q1dd[rr], qc, wbot);
                        val = val - div0(f5t - f5b, r_DJR[rr]);
                    } else if (L == 0) {
                        const float f5t = flux1(qc, AT(sQc, lx, ly), wtop);
                        val = val - div0(f5t, r_DJR[rr]);
                    } else {
                        const float f5b = flux1(r_q1dd[rr], qc, wbot);
                        val = val - div0(qc * wtop - f5b, r_DJR[rr]);
                    }
                    outg[ix(g, i, L, j)] = val;
                }
            }
        }

        // ---------------- rotate the per-cell z state ------------------------
        if (haveA) {
#pragma unroll
            for (int rr = 0; rr < RPW; rr++) {
                const int ly = warp + NW * rr + 2, lx = lane + 2;
                const int i = max(min(i0 - 2 + lx, nx - 1), 0), j = min(j0 - 2 + ly, ny - 1);
                r_q1dd[rr] = r_q1dn[rr];
                r_q1dn[rr] = AT(sQc, lx, ly);   // q1 at level t, "below" for level t+1
                r_q0dn[rr] = AT(sQ0c, lx, ly);
                r_fz[rr] = n_fz[rr];
                r_w2[rr] = n_w2[rr];
                r_bzi[rr] = n_bzi[rr];
                r_bzo[rr] = n_bzo[rr];
                r_w2l[rr] = n_w2l[rr];
                r_part[rr] = n_part[rr];
                r_DJR[rr] = DJR[ix(g, i, t, j)];
            }
        }
    }
    __syncthreads();  // the CTA may start another tile in the same shared memory
#undef AT
}

template <bool FCT, class SH>
__global__ void __launch_bounds__(SH::NT, (SH::NT <= 128 ? 5 : SH::NT <= 256 ? 3 : SH::NT <= 512 ? 2 : 1))
    k_mp_corr(Geo g, SpeciesPtrs sp, int nspecies, int tiles_x, const float *__restrict__ Um,
              const float *__restrict__ Vm, const float *__restrict__ Wp, const float *__restrict__ Gc,
              const float *__restrict__ DJR, const float *__restrict__ dz)
{
    extern __shared__ float4 sm4[];
    const int s = blockIdx.x % nspecies;
    const int tile = blockIdx.x / nspecies;
    const int i0 = (tile % tiles_x) * mpf::TX - 2;  // first output column; i0-2 is a multiple of 4
    const int j0 = 1 + (tile / tiles_x) * SH::TY;
    mp_corr_tile<FCT, SH>(reinterpret_cast<float *>(sm4), g, sp.q0[s], sp.q1[s], sp.out[s], i0, j0, Um, Vm, Wp, Gc,
                          DJR, dz);
}

inline bool fused_eligible(int order, int fct) { return order == 2 && (fct == 0 || fct == 1); }

// tile tx covers output columns [TX*tx-2, TX*tx+TX-2); the last must reach nx-2
inline int mp_tiles_x(const Geo &g) { return g.nx / mpf::TX + 1; }
inline int mp_tiles_y(const Geo &g, int ty) { return (g.ny - 2 + ty - 1) / ty; }

// Debug check (parameters%debug): flags any interior cell whose donor-cell
// outflow fraction, sum of outgoing Courant fluxes over J*rho (dz*J*rho for
// the vertical faces), exceeds 1.
__global__ void k_courant(Geo g, const float *__restrict__ Um, const float *__restrict__ Vm,
                          const float *__restrict__ Wm, const float *__restrict__ dz, const float *__restrict__ jaco,
                          const float *__restrict__ rho, int use_rho, int *__restrict__ flag)
{
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    int i = (int)(t % (size_t)g.nx);
    size_t rest = t / (size_t)g.nx;
    int k = (int)(rest % (size_t)g.nz);
    int j = (int)(rest / (size_t)g.nz);
    if (j >= g.ny || i == 0 || i == g.nx - 1 || j == 0 || j == g.ny - 1) return;
    size_t c = ix(g, i, k, j), sy = (size_t)g.P * g.nz, sz = (size_t)g.P;
    float r = use_rho ? rho[c] : 1.0f;
    float h = (fmaxf(0.0f, Um[c + 1]) - fminf(0.0f, Um[c]) + fmaxf(0.0f, Vm[c + sy]) - fminf(0.0f, Vm[c])) /
              (jaco[c] * r);
    float wb = k > 0 ? Wm[c - sz] : 0.0f;
    float v = (fmaxf(0.0f, Wm[c]) - fminf(0.0f, wb)) / (dz[c] * jaco[c] * r);
    if (!(h + v <= 1.0f)) atomicExch(flag, 1);
}

inline int check_courant(cudaStream_t st, const Geo &g, const float *Um, const float *Vm, const float *Wm,
                         const float *dz, const float *jaco, const float *rho, int use_rho)
{
    int *flag = nullptr;
    int host = 0;
    if (cudaMallocAsync(&flag, sizeof(int), st) != cudaSuccess) return 1;
    cudaMemsetAsync(flag, 0, sizeof(int), st);
    size_t n = (size_t)g.nx * g.nz * g.ny;
    k_courant<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, Um, Vm, Wm, dz, jaco, rho, use_rho, flag);
    cudaMemcpyAsync(&host, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(flag, st);
    cudaStreamSynchronize(st);
    return host;
}

}  // namespace icar

namespace icar {

// Tile shapes of the fused correction kernel (selected per grid shape by
// the autotuner): output rows per tile and warps per CTA.
using MpShape8 = mpf::Shape<8, 4>;
using MpShape16 = mpf::Shape<15, 16>;
using MpShape24 = mpf::Shape<24, 8>;
using MpShape32 = mpf::Shape<31, 32>;
constexpr int MP_NSHAPES = 4;
inline int mp_shape_ty(int shape)
{
    const int ty[MP_NSHAPES] = {8, 15, 24, 31};
    return ty[shape < 0 || shape >= MP_NSHAPES ? 1 : shape];
}

template <class SH>
inline cudaError_t mp_corr_attr()
{
    cudaError_t e = cudaFuncSetAttribute(k_mp_corr<true, SH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)mpf::smem_bytes<SH>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mp_corr<false, SH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)mpf::smem_bytes<SH>());
    return e;
}

// Allow every instantiation its dynamic shared memory (once per device).
inline cudaError_t mp_corr_setup()
{
    cudaError_t e = cudaFuncSetAttribute(k_mp_upwind_cols, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)upf::SMEM);
    if (e == cudaSuccess) e = mp_corr_attr<MpShape8>();
    if (e == cudaSuccess) e = mp_corr_attr<MpShape16>();
    if (e == cudaSuccess) e = mp_corr_attr<MpShape24>();
    if (e == cudaSuccess) e = mp_corr_attr<MpShape32>();
    return e;
}

template <class SH>
inline void mp_corr_launch_t(cudaStream_t st, const Geo &g, const SpeciesPtrs &sp, int S, int fct, const float *Um,
                             const float *Vm, const float *Wp, const float *Gc, const float *DJR, const float *dz)
{
    const int tx = mp_tiles_x(g), ty = mp_tiles_y(g, SH::TY);
    const unsigned nblk = (unsigned)(tx * ty * S);
    if (fct)
        k_mp_corr<true, SH><<<nblk, SH::NT, mpf::smem_bytes<SH>(), st>>>(g, sp, S, tx, Um, Vm, Wp, Gc, DJR, dz);
    else
        k_mp_corr<false, SH><<<nblk, SH::NT, mpf::smem_bytes<SH>(), st>>>(g, sp, S, tx, Um, Vm, Wp, Gc, DJR, dz);
}

inline void mp_corr_launch(cudaStream_t st, int shape, const Geo &g, const SpeciesPtrs &sp, int S, int fct,
                           const float *Um, const float *Vm, const float *Wp, const float *Gc, const float *DJR,
                           const float *dz)
{
    switch (shape) {
    case 0: mp_corr_launch_t<MpShape8>(st, g, sp, S, fct, Um, Vm, Wp, Gc, DJR, dz); break;
    case 2: mp_corr_launch_t<MpShape24>(st, g, sp, S, fct, Um, Vm, Wp, Gc, DJR, dz); break;
    case 3: mp_corr_launch_t<MpShape32>(st, g, sp, S, fct, Um, Vm, Wp, Gc, DJR, dz); break;
    default: mp_corr_launch_t<MpShape16>(st, g, sp, S, fct, Um, Vm, Wp, Gc, DJR, dz); break;
    }
}

}  // namespace icar
