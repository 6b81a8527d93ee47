// Single-pass MPDATA step (mpdata_order 2, FCT on or off): one launch per
// advect call for every species, each CTA one 56 x 26 column tile of one
// species marching up the column.  Per level it
//
//   P0  recomputes the donor-cell pass q0 -> q1 one level ahead on the tile
//       plus a two-cell halo (upwind_advection, adv_mpdata.f90:43-103), so
//       q1 never goes through HBM;
//   P1  forms the antidiffusive pseudo-velocities u2, v2, w2 with their
//       cross terms (mpdata_fluxes, adv_mpdata.f90:105-252), scaled by 0.5
//       and 0.5*dz (:378-380);
//   P2  forms the FCT limiter's per-cell bounds, in/out flux sums and beta
//       factors in x, y and z (flux_limiter, adv_mpdata.f90:254-350, in the
//       per-cell form of adv_mpdata_FCT_core.f90:47-116, first and last cells
//       of every line included);
//   P3  limits each face with the betas of the two cells beside it and
//       applies the corrective donor-cell pass (adv_mpdata.f90:384): the
//       horizontal part at this level, the vertical part one level down.
//
// Data movement.  The level planes of q0 and of the per-step fields (U_m,
// V_m, W_m/dz, J*rho) arrive in shared memory by TMA (64 x 32 boxes of
// this GPU's own arrays, each CTA loading its own) one level ahead of use,
// completing on mbarriers; W_m, dz*J*rho and dz of the thread's own columns
// come by plain
// loads one level ahead.  Each thread owns an x-pair of columns in two rows
// and works on the pair with packed f32x2 arithmetic; x neighbours come by
// warp shuffles, y neighbours from the shared planes.
//
// Arithmetic.  EXACT = true evaluates the reference's FP32 expressions in
// their order with IEEE division and no contraction (the translation unit is
// built with -fmad=false), so results equal the CPU oracle bit for bit.
// EXACT = false (the fast variant) rewrites the same scheme for throughput:
// reciprocals by the hardware approximation, fused multiply-adds, donor-cell
// fluxes as U * (U > 0 ? l : r), and each face's pair sums shared between
// its ratio and cross terms; its results differ from the exact ones by
// rounding only (the tolerance is stated by the tests).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "common.cuh"
#include "tma.cuh"

namespace icar {

namespace op {
constexpr int PW = 64;               // plane width (floats): x from x0 to x0+63
constexpr int PH = 32;               // plane rows: y from j0-3 to j0+28
constexpr int NW = 16;               // warps per CTA
constexpr int NT = NW * 32;
constexpr int RPW = PH / NW;         // rows per warp (warp w owns rows w and w+NW)
constexpr int TX = PW - 8;           // 56 output columns of an inner column tile: plane x 4..59
constexpr int TY = PH - 6;           // 26 output rows: plane y 3..28
constexpr int PLANE = PW * PH;
constexpr uint32_t PLANE_BYTES = PLANE * sizeof(float);
// TMA-filled slots (ring index = level mod ring length)
constexpr int S_Q0 = 0;              // q0, 5 levels (t-1 .. t+3)
constexpr int S_U = 5;               // U_m, 3 levels
constexpr int S_V = 8;               // V_m, 3 levels
constexpr int S_WP = 11;             // W_m/dz, 3 levels
constexpr int S_G = 14;              // J*rho, 3 levels
// thread-written slots
constexpr int S_Q1 = 17;             // q1, 5 levels (t-3 .. t+1)
constexpr int S_V2 = 22;             // unlimited v2 of the current level
constexpr int S_BYI = 23, S_BYO = 24;  // y-limiter betas of the current level
constexpr int NPLANES = 25;
constexpr size_t SMEM = (size_t)NPLANES * PLANE * sizeof(float) + 128;
constexpr uint64_t WAIT_NS = 2000000000ull;  // a TMA wait gives up after 2 s
constexpr int MAXS = 32;             // species per launch

// Column tiles.  An inner tile's plane keeps 4 halo columns on each side
// (56 output columns; the plane origin stays 16-byte aligned for TMA).  The
// first and last tiles of a row sit on the domain's edges, where there is
// nothing to read beyond the edge, so the first outputs the 60 columns from
// x = 0 and the last ends at the domain's last column: nx = 512 takes 9
// tiles where 56-column tiling takes 10.
__host__ __device__ inline int tiles_x(int nx) { return nx <= PW ? 1 : 2 + max(0, (nx - 120 + TX - 1) / TX); }

// Plane origin x0 and output columns [xlo, xhi) (plane coordinates) of
// column tile tx of ntx.
__device__ __forceinline__ void xtile(int nx, int tx, int ntx, int &x0, int &xlo, int &xhi)
{
    if (ntx == 1) {
        x0 = 0, xlo = 0, xhi = nx;
    } else if (tx == 0) {
        x0 = 0, xlo = 0, xhi = PW - 4;
    } else {
        const int start = PW - 4 + TX * (tx - 1);   // first output column
        if (tx < ntx - 1) {
            x0 = start - 4, xlo = 4, xhi = PW - 4;
        } else {
            x0 = (nx - PW + 3) & ~3;               // the plane reaches the last column (at most 3 beyond)
            xlo = start - x0, xhi = nx - x0;
        }
    }
}
}  // namespace op

// Kernel parameters.  The tensor maps (64 x 1 x 32 boxes over (x, z, y))
// live in a device table (cudaMalloc'd, so every 128-byte map is 64-byte
// aligned as TMA requires): q0maps[s] for the species inputs, fmaps[0..3]
// for U_m, V_m, W_m/dz and J*rho.
struct OnePassParams {
    const CUtensorMap *q0maps;
    const CUtensorMap *fmaps;
    float *out[op::MAXS];
    const float *Wm, *DJR, *dz;
    int *err;            // 1: a TMA wait gave up; 2: a TMA operand was misaligned (loads skipped)
    Geo g;
    int nspecies;
    int tiles_x;
};

namespace opx {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ float2 ld2(const float *plane, int Y, int X)
{
    return *reinterpret_cast<const float2 *>(plane + Y * op::PW + X);
}
__device__ __forceinline__ void st2(float *plane, int Y, int X, float2 v)
{
    *reinterpret_cast<float2 *>(plane + Y * op::PW + X) = v;
}
__device__ __forceinline__ float up(float v) { return __shfl_up_sync(FULL, v, 1); }     // lane-1's value
__device__ __forceinline__ float dn(float v) { return __shfl_down_sync(FULL, v, 1); }   // lane+1's value
// the pair shifted one cell left (x-1, x) / right (x+1, x+2)
__device__ __forceinline__ float2 lft(float2 v) { return make_float2(up(v.y), v.x); }
__device__ __forceinline__ float2 rgt(float2 v) { return make_float2(v.y, dn(v.x)); }

// Hardware reciprocal approximation, flushing subnormal operands and results.
// Every divisor of the fast variant is a metric term (J*rho, dz*J*rho and
// their face sums), a sum of tracer values plus 1e-10, or a flux sum plus
// 1e-15: none is subnormal or above 2^126, so flushing changes no result,
// and it spares the multi-instruction subnormal handling around each
// reciprocal that the non-flushing form needs.
__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;\n" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float2 rcp2(float2 b) { return make_float2(rcp_approx(b.x), rcp_approx(b.y)); }
__device__ __forceinline__ float2 div2x(float2 a, float2 b) { return make_float2(a.x / b.x, a.y / b.y); }

// donor-cell flux, exact form ((U+|U|)*l + (U-|U|)*r)/2 (adv_mpdata.f90:23-41)
__device__ __forceinline__ float2 flux_x(float2 l, float2 r, float2 U)
{
    const float2 a = abs2(U);
    return mul2x(add2x(mul2x(add2x(U, a), l), mul2x(sub2x(U, a), r)), splat2(0.5f));
}
// the same flux as U times the upwind value (equal but for rounding of
// subnormal products)
__device__ __forceinline__ float2 flux_f(float2 l, float2 r, float2 U)
{
    return mul2(U, make_float2(U.x > 0.0f ? l.x : r.x, U.y > 0.0f ? l.y : r.y));
}
// pair arithmetic of the variant: exact (never contracted) or packed
template <bool EXACT>
__device__ __forceinline__ float2 ad(float2 a, float2 b)
{
    if constexpr (EXACT) return add2x(a, b);
    else return add2(a, b);
}
template <bool EXACT>
__device__ __forceinline__ float2 sb(float2 a, float2 b)
{
    if constexpr (EXACT) return sub2x(a, b);
    else return sub2(a, b);
}
template <bool EXACT>
__device__ __forceinline__ float2 ml(float2 a, float2 b)
{
    if constexpr (EXACT) return mul2x(a, b);
    else return mul2(a, b);
}

template <bool EXACT>
__device__ __forceinline__ float2 flux(float2 l, float2 r, float2 U)
{
    if constexpr (EXACT) return flux_x(l, r, U);
    else return flux_f(l, r, U);
}

// FCT beta num/den (den > 0): min(1, num/den) as the reference uses it; a
// quotient >= 1 is returned as 1 without dividing, num == 0 gives 0.
template <bool EXACT>
__device__ __forceinline__ float beta(float num, float den)
{
    if constexpr (EXACT) {
        if (num >= den) return 1.0f;
        if (num == 0.0f) return 0.0f;
        return num / den;
    } else {
        return fminf(1.0f, num * rcp_approx(den));
    }
}

// Limited pseudo-velocity at a face (adv_mpdata_FCT_core.f90:103-115).
// The fast variant's betas are already at most 1, and its form is a select.
template <bool EXACT>
__device__ __forceinline__ float limit(float u, float bin_r, float bout_l, float bin_l, float bout_r)
{
    if constexpr (EXACT) {
        if (u > 0.0f) return fminf(fminf(1.0f, bin_r), bout_l) * u;
        if (u < 0.0f) return fminf(fminf(1.0f, bin_l), bout_r) * u;
        return u;
    } else {
        return (u > 0.0f ? fminf(bin_r, bout_l) : fminf(bin_l, bout_r)) * u;
    }
}

// Limited flux through a pair of faces in the fast variant: the face
// velocity u times the limiter factor of its sign (min(bin_r, bout_l) for
// u > 0, min(bin_l, bout_r) otherwise) times the upwind cell's value; one
// comparison per face serves both selects.
__device__ __forceinline__ float2 lim_flux2(float2 u, float2 ql, float2 qr, float2 bin_r, float2 bout_l, float2 bin_l,
                                            float2 bout_r)
{
    const bool px = u.x > 0.0f, py = u.y > 0.0f;
    const float2 b = make_float2(fminf(px ? bin_r.x : bin_l.x, px ? bout_l.x : bout_r.x),
                                 fminf(py ? bin_r.y : bin_l.y, py ? bout_l.y : bout_r.y));
    const float2 q = make_float2(px ? ql.x : qr.x, py ? ql.y : qr.y);
    return mul2(mul2(u, b), q);
}

// Per-cell limiter terms of one direction (the carried form of the FCT
// sweep): bounds over the cell and its two line neighbours, in/out flux sums
// from the fluxes on its two faces, with the reference's first/last-cell
// cases.  pos: 0 interior, 1 first cell, 2 last cell.  w lines (flux_is_w)
// keep the end fluxes; x/y lines use 0 there.
template <bool EXACT>
__device__ __forceinline__ void fct_cell(float q1m, float q1c, float q1p, float q0m, float q0c, float q0p, float fl,
                                         float fr, int pos, bool wline, float &bin, float &bout)
{
    float qmax, qmin, fin, fout;
    if (pos == 1) {
        qmax = fmaxf(fmaxf(q1c, q1p), fmaxf(q0c, q0p));
        qmin = fminf(fminf(q1c, q1p), fminf(q0c, q0p));
        if (wline) {
            fin = 0.0f - fminf(0.0f, fr);
            fout = fmaxf(0.0f, fr);
        } else {
            fin = 0.0f;
            fout = 0.0f;
        }
    } else if (pos == 2) {
        qmax = fmaxf(fmaxf(q1m, q1c), q0m);
        qmin = fminf(fminf(q1m, q1c), q0m);
        if (wline) {
            fin = fmaxf(0.0f, fl) - fminf(0.0f, fl);
            fout = fin;
        } else {
            fin = 0.0f;
            fout = 0.0f;
        }
    } else {
        qmax = fmaxf(fmaxf(fmaxf(q1m, q1c), q1p), fmaxf(fmaxf(q0m, q0c), q0p));
        qmin = fminf(fminf(fminf(q1m, q1c), q1p), fminf(fminf(q0m, q0c), q0p));
        fin = fmaxf(0.0f, fl) - fminf(0.0f, fr);
        fout = fmaxf(0.0f, fr) - fminf(0.0f, fl);
    }
    const float e15 = 1e-15f;
    bin = beta<EXACT>(qmax - q1c, fin + e15);
    bout = beta<EXACT>(q1c - qmin, fout + e15);
}

// The same terms for a pair of interior cells (pos 0) in the fast
// variant's packed arithmetic.
__device__ __forceinline__ void fct_pair_fast(float2 q1m, float2 q1c, float2 q1p, float2 q0m, float2 q0c, float2 q0p,
                                              float2 fl, float2 fr, float2 &bin, float2 &bout)
{
    const float2 qmax = make_float2(fmaxf(fmaxf(fmaxf(q1m.x, q1c.x), q1p.x), fmaxf(fmaxf(q0m.x, q0c.x), q0p.x)),
                                    fmaxf(fmaxf(fmaxf(q1m.y, q1c.y), q1p.y), fmaxf(fmaxf(q0m.y, q0c.y), q0p.y)));
    const float2 qmin = make_float2(fminf(fminf(fminf(q1m.x, q1c.x), q1p.x), fminf(fminf(q0m.x, q0c.x), q0p.x)),
                                    fminf(fminf(fminf(q1m.y, q1c.y), q1p.y), fminf(fminf(q0m.y, q0c.y), q0p.y)));
    const float2 fin = sub2(make_float2(fmaxf(0.0f, fl.x), fmaxf(0.0f, fl.y)),
                            make_float2(fminf(0.0f, fr.x), fminf(0.0f, fr.y)));
    const float2 fout = sub2(make_float2(fmaxf(0.0f, fr.x), fmaxf(0.0f, fr.y)),
                             make_float2(fminf(0.0f, fl.x), fminf(0.0f, fl.y)));
    const float2 e15 = splat2(1e-15f);
    const float2 a = mul2(sub2(qmax, q1c), rcp2(add2(fin, e15)));
    const float2 b = mul2(sub2(q1c, qmin), rcp2(add2(fout, e15)));
    bin = make_float2(fminf(1.0f, a.x), fminf(1.0f, a.y));
    bout = make_float2(fminf(1.0f, b.x), fminf(1.0f, b.y));
}

// The first and last cells of an x or y line in the fast variant, as the
// interior form on substituted operands: a neighbour the reference's bounds
// leave out takes a value already in them (the first cell's bounds omit the
// cell before it; the last cell's take q1 of the cell before it and of
// itself and q0 of the cell before it only), and both fluxes are zero (the
// x and y lines carry no flux sums at their ends).
__device__ __forceinline__ void fct_edge_sub(bool first, bool last, float &q1m, float q1c, float &q1p, float &q0m,
                                             float &q0c, float &q0p, float &fl, float &fr)
{
    if (first) {
        q1m = q1c;
        q0m = q0c;
    }
    if (last) {
        q1p = q1c;
        q0c = q0m;
        q0p = q0m;
    }
    if (first || last) fl = fr = 0.0f;
}

// Cross-term ratio (((a-b)+c)-d) / (den + 1e-10) with the reference's
// operand order for the denominator chosen by the caller.
__device__ __forceinline__ float2 xnum(float2 a, float2 b, float2 c, float2 d) { return sub2x(add2x(sub2x(a, b), c), d); }
__device__ __forceinline__ float2 xden(float2 p, float2 q, float2 r, float2 s)
{
    return add2x(add2x(add2x(add2x(p, q), r), s), splat2(1e-10f));
}
// 0.25 * (((a + b) + c) + d)
__device__ __forceinline__ float2 avg4(float2 a, float2 b, float2 c, float2 d)
{
    return mul2x(splat2(0.25f), add2x(add2x(add2x(a, b), c), d));
}

// Pseudo-velocity of a face, exact form: |U|(1-|U|/(0.5*Gs)) (r-l)/(r+l+eps)
__device__ __forceinline__ float2 base_x(float2 U, float2 Gs, float2 r, float2 l)
{
    const float2 a = abs2(U);
    float2 v = mul2x(a, sub2x(splat2(1.0f), div2x(a, mul2x(splat2(0.5f), Gs))));
    return div2x(mul2x(v, sub2x(r, l)), add2x(add2x(r, l), splat2(1e-10f)));
}
// minus the cross term 0.5*U*ev*eq/Gs, exact form
__device__ __forceinline__ float2 cross_x(float2 v, float2 U, float2 ev, float2 eq, float2 Gs)
{
    return sub2x(v, div2x(mul2x(mul2x(mul2x(splat2(0.5f), U), ev), eq), Gs));
}

}  // namespace opx

// One tile's march.  INT: the whole 64 x 32 plane lies inside the domain's
// interior (x in [1, nx-2], y in [1, ny-2]), so no cell of the tile meets a
// domain edge: the edge cases of the reference (boundary ring, first/last
// cells of the limiter lines, faces that do not exist) drop out at compile
// time.  Tiles that touch an edge take the general form.
// bars: two mbarriers initialised once per CTA; ph[0], ph[1] count the
// phases each has completed so far (a CTA may run several tiles), and are
// advanced here by the phases this tile completes.  Returns false when a
// TMA wait gave up (the flag in p.err is then set and the CTA must stop).
template <bool EXACT, bool FCT, bool INT>
__device__ __forceinline__ bool onepass_tile(float *sm, uint64_t *bars, uint32_t *ph, const OnePassParams &p, int s,
                                             int x0, int xlo, int xhi, int j0)
{
    using namespace op;
    using namespace opx;
    const Geo g = p.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int y0 = j0 - 3;
    // the warp index through a shuffle from lane 0, so that the compiler
    // treats every row condition below as warp-uniform (plain branches, no
    // reconvergence bookkeeping)
    const int lane = threadIdx.x & 31, warp = __shfl_sync(0xffffffffu, (int)(threadIdx.x >> 5), 0);
    const int X = 2 * lane;
    const int ia = x0 + X, ib = ia + 1;   // global x of the pair
    const CUtensorMap *mq = p.q0maps + s;
    const CUtensorMap *mU = p.fmaps, *mV = p.fmaps + 1, *mW = p.fmaps + 2, *mG = p.fmaps + 3;
    float *__restrict__ outg = p.out[s];
    auto P = [&](int slot) { return sm + (size_t)slot * PLANE; };
    auto sq0 = [&](int l) { return P(S_Q0 + (l + 5) % 5); };       // level -1 maps to a valid slot
    auto sU = [&](int l) { return P(S_U + l % 3); };
    auto sV = [&](int l) { return P(S_V + l % 3); };
    auto sW = [&](int l) { return P(S_WP + (l + 3) % 3); };   // level -1 maps to a valid slot
    auto sG = [&](int l) { return P(S_G + l % 3); };
    auto sQ1 = [&](int l) { return P(S_Q1 + (l + 5) % 5); };       // levels -2, -1 map to valid slots

    // ---- TMA issue: the loads a level adds (elected thread only)
    // TMA operands must be aligned (map 64 B, destination 128 B, barrier
    // 8 B); a misaligned one is reported (flag 2) and its batch is skipped,
    // so the CTA finishes instead of faulting
    auto tma_ok = [&](uint64_t *bar) {
        const bool good = (((uintptr_t)mq | (uintptr_t)p.fmaps) & 63u) == 0 && (smem_u32(sm) & 127u) == 0 &&
                          (smem_u32(bar) & 7u) == 0;
        if (!good) atomicExch(p.err, 2);
        return good;
    };
    auto issue = [&](uint64_t *bar, int lq0, int lu, int lv, int lw, int lg) {
        if (!tma_ok(bar)) {
            mbar_arrive_expect_tx(bar, 0);
            return;
        }
        uint32_t n = 0;
        n += lq0 < nz;
        n += lu < nz;
        n += lv < nz;
        n += (lw >= 0 && lw < nz);
        n += lg < nz;
        mbar_arrive_expect_tx(bar, n * PLANE_BYTES);
        if (lq0 < nz) tma_load_3d(sq0(lq0), mq, x0, lq0, y0, bar);
        if (lu < nz) tma_load_3d(sU(lu), mU, x0, lu, y0, bar);
        if (lv < nz) tma_load_3d(sV(lv), mV, x0, lv, y0, bar);
        if (lw >= 0 && lw < nz) tma_load_3d(sW(lw), mW, x0, lw, y0, bar);
        if (lg < nz) tma_load_3d(sG(lg), mG, x0, lg, y0, bar);
    };
    bool ok = true;
    // The batch waited for at iteration t was issued on bars[t & 1]: the
    // prologue's on bars[0], iteration t-1's otherwise.  Its phase number is
    // the barrier's count at tile start plus the batches issued on it since.
    const uint32_t b0 = ph[0], b1 = ph[1];
    auto phase_of = [&](int t) -> uint32_t { return (t & 1) ? b1 + (uint32_t)(t - 1) / 2 : b0 + (uint32_t)t / 2; };
    // bounded wait on the batch of iteration t, by every thread; a thread
    // whose wait gave up raises the flag and reports false (the CTA then
    // agrees at its next barrier to stop, after draining with a bound what
    // it issued)
    auto wait_mine = [&](int t) {
        const bool mine = mbar_wait_bounded(&bars[t & 1], phase_of(t) & 1u, WAIT_NS);
        if (!mine) atomicExch(p.err, 1);
        return mine;
    };
    // every batch completes a phase (one arrival, possibly zero bytes): the
    // prologue and the odd iterations on bars[0], the even ones on bars[1]
    ph[0] = b0 + 1 + (uint32_t)(nz + 1) / 2;
    ph[1] = b1 + (uint32_t)nz / 2 + 1;

    if (threadIdx.x == 0) tma_prefetch_map(mq);
    if (threadIdx.x == 0) {
        // iteration 0 (and the level-0 donor pass before it) needs q0 at
        // levels 0..2, U_m, V_m and J*rho at 0..1 and W_m/dz at 0 (nz >= 3)
        uint32_t cnt = 0;
        for (int l = 0; l < 3; l++) cnt += l < nz;
        for (int l = 0; l < 2; l++) cnt += 3 * (l < nz);
        cnt += 1;
        const bool good = tma_ok(&bars[0]);
        mbar_arrive_expect_tx(&bars[0], good ? cnt * PLANE_BYTES : 0u);
        for (int l = 0; good && l < 3; l++)
            if (l < nz) tma_load_3d(sq0(l), mq, x0, l, y0, &bars[0]);
        for (int l = 0; good && l < 2; l++) {
            if (l >= nz) continue;
            tma_load_3d(sU(l), mU, x0, l, y0, &bars[0]);
            tma_load_3d(sV(l), mV, x0, l, y0, &bars[0]);
            tma_load_3d(sG(l), mG, x0, l, y0, &bars[0]);
        }
        if (good) tma_load_3d(sW(0), mW, x0, 0, y0, &bars[0]);
    }

    // ---- per-row constants and carried state --------------------------
    int rowY[RPW], rowj[RPW];
    size_t rowc[RPW];      // global offset of (ia, level 0, j) (clamped into the array)
    bool rowin[RPW];       // row inside the domain
#pragma unroll
    for (int r = 0; r < RPW; r++) {
        rowY[r] = warp + NW * r;
        rowj[r] = y0 + rowY[r];
        rowin[r] = rowj[r] >= 0 && rowj[r] < ny;
        const int ci = max(min(ia, g.P - 2), 0), cj = max(min(rowj[r], ny - 1), 0);
        rowc[r] = ix(g, ci, 0, cj);
    }
    const bool inA = ia >= 0 && ia < nx, inB = ib >= 0 && ib < nx;
    const size_t lstride = (size_t)g.P;

    // own-column values by plain loads, one level ahead
    // (the fast variant carries dz*J*rho as its reciprocal: each value
    // divides twice, in the donor pass and in the corrective pass)
    float2 r_wm[RPW], n_wm[RPW], r_djr0[RPW], r_djrm[RPW], n_djr[RPW], n_dz[RPW];
    auto djr_in = [](float2 v) -> float2 {
        if constexpr (EXACT) return v;
        else return rcp2(v);
    };
    // carried z state of the output cells, the donor pass's flux through
    // the top of the level it formed last, and (fast variant) the
    // reciprocal of J*rho that the donor pass formed for the level the
    // corrective pass updates next (r_rg: level t, n_rg: level t+1)
    float2 r_w2[RPW], r_bzi[RPW], r_bzo[RPW], r_fb[RPW], r_part[RPW], r_vt[RPW], r_rg[RPW], n_rg[RPW];
    auto ldcol = [&](const float *src, int r, int lev) -> float2 {
        return *reinterpret_cast<const float2 *>(src + rowc[r] + (size_t)lev * lstride);
    };
#pragma unroll
    for (int r = 0; r < RPW; r++) {
        r_wm[r] = ldcol(p.Wm, r, 0);
        r_djr0[r] = djr_in(ldcol(p.DJR, r, 0));
        n_wm[r] = nz > 1 ? ldcol(p.Wm, r, 1) : splat2(0.0f);
        n_djr[r] = nz > 1 ? ldcol(p.DJR, r, 1) : splat2(1.0f);
        n_dz[r] = ldcol(p.dz, r, 0);
        r_djrm[r] = splat2(1.0f);
        r_w2[r] = r_bzi[r] = r_bzo[r] = r_fb[r] = r_part[r] = r_vt[r] = splat2(0.0f);
    }

    const float2 zero2 = splat2(0.0f);

    // ---- P0: donor-cell pass at level L into the q1 plane of L ----------
    // wtop = W_m(L), djr = dz*J*rho at L (its reciprocal in the fast
    // variant), own pair.  Levels are formed in order, so the flux through
    // the bottom of L is the one through the top of L-1, carried in r_vt.
    auto donor = [&](int L, int r, float2 wtop, float2 djr) {
        const int Y = rowY[r], j = rowj[r];
        const bool need = Y >= 1 && Y <= PH - 2;     // warp-uniform
        if (!need) return;
        const float *Q = sq0(L);
        const float2 c = ld2(Q, Y, X);
        const float2 n = ld2(Q, Y + 1, X), sth = ld2(Q, Y - 1, X);
        const float2 w = lft(c);
        const float2 uw = ld2(sU(L), Y, X);
        const float2 vs = ld2(sV(L), Y, X), vn = ld2(sV(L), Y + 1, X);
        const float2 G = ld2(sG(L), Y, X);
        // a cell's east face is the next cell's west face: same operands,
        // same value, so it is formed once and passed along by a shuffle
        const float2 fw = flux<EXACT>(w, c, uw), fe = rgt(fw);
        const float2 f3 = flux<EXACT>(c, n, vn), f4 = flux<EXACT>(sth, c, vs);
        const float2 hd = ad<EXACT>(sb<EXACT>(fe, fw), sb<EXACT>(f3, f4));
        float2 val;
        const bool mid = L > 0 && L < nz - 1;
        float2 vt = zero2;
        const float2 vb = L > 0 ? r_vt[r] : zero2;
        if (L < nz - 1) vt = flux<EXACT>(c, ld2(sq0(L + 1), Y, X), wtop);
        r_vt[r] = vt;
        if constexpr (EXACT) {
            val = sub2x(c, div2x(hd, G));
            if (mid) val = sub2x(val, div2x(sub2x(vt, vb), djr));
            else if (L == 0) val = sub2x(val, div2x(vt, djr));
            else val = sub2x(val, div2x(sub2x(mul2x(c, wtop), vb), djr));
        } else {
            const float2 vdiv = mid ? sub2(vt, vb) : (L == 0 ? vt : sub2(mul2(c, wtop), vb));
            const float2 rg = rcp2(G);
            n_rg[r] = rg;
            val = sub2(sub2(c, mul2(hd, rg)), mul2(vdiv, djr));
        }
        float2 q1 = val;
        if (!INT) {
            const bool jin = j >= 0 && j < ny, jring = j == 0 || j == ny - 1;
            q1.x = !(inA && jin) ? 0.0f : ((jring || ia == 0 || ia == nx - 1) ? c.x : val.x);
            q1.y = !(inB && jin) ? 0.0f : ((jring || ib == 0 || ib == nx - 1) ? c.y : val.y);
        }
        st2(sQ1(L), Y, X, q1);
    };

    // ---- prologue: batch 0 landed -> q1 at level 0 ----------------------
    ok = __syncthreads_and(wait_mine(0) ? 1 : 0) != 0;
    if (!ok) goto drain;
#pragma unroll
    for (int r = 0; r < RPW; r++) donor(0, r, r_wm[r], r_djr0[r]);

    // Three block barriers per level: after P0, after P1 (v2 plane), after
    // P2 (y betas).  P0 of iteration t may overlap P3 of iteration t-1: it
    // writes the q1 slot of level t+1, which the 5-level ring keeps apart
    // from the levels t-3 .. t-1 that P3 reads, and reads only TMA planes.
    for (int t = 0; t <= nz; t++) {
        const bool landed = t == 0 || wait_mine(t);

        const bool haveA = t < nz;
        // own-column values for this iteration; prefetch the next level's
        float2 c_wmn[RPW], c_djrn[RPW], c_dz[RPW];
#pragma unroll
        for (int r = 0; r < RPW; r++) {
            c_wmn[r] = n_wm[r];
            c_djrn[r] = djr_in(n_djr[r]);
            r_rg[r] = n_rg[r];
            c_dz[r] = n_dz[r];
            if (t + 2 < nz) {
                n_wm[r] = ldcol(p.Wm, r, t + 2);
                n_djr[r] = ldcol(p.DJR, r, t + 2);
            }
            if (t + 1 < nz) n_dz[r] = ldcol(p.dz, r, t + 1);
        }

        // ---- P0: q1 at level t+1 ------------------------------------------
        if (t + 1 < nz) {
#pragma unroll
            for (int r = 0; r < RPW; r++) donor(t + 1, r, c_wmn[r], c_djrn[r]);
        }
        // every thread is past iteration t-1 and the batch of iteration t
        // landed (or the CTA stops): the planes that batch t+1 overwrites
        // (q0 of t-2, U_m, V_m, J*rho of t-1, W_m/dz of t-2) are free.  The
        // elected thread's warp has one row with nothing to do in P1, so
        // the issue costs no time on the block's critical path.
        ok = __syncthreads_and(landed ? 1 : 0) != 0;
        if (!ok) goto drain;
        if (threadIdx.x == 0) issue(&bars[(t + 1) & 1], t + 3, t + 2, t + 2, t + 1, t + 2);

        float2 u2[RPW], v2[RPW], w2[RPW], fz[RPW];
        float2 bxi[RPW], bxo[RPW], byi[RPW], byo[RPW], bzi[RPW], bzo[RPW];
        if (haveA) {
            const bool kint = t > 0 && t < nz - 1;
            const bool top = t == nz - 1;
            // ---- P1: pseudo-velocities at level t ---------------------------
            // Each face block loads its own stencil (shared-memory loads are
            // cheap; long live ranges across the three blocks are not).
            const float *Qc = sQ1(t), *Qu = sQ1(t + 1), *Qd = sQ1(t - 1);
            const float *Uc = sU(t), *Uup = sU(t + 1), *Vc = sV(t), *Vup = sV(t + 1);
            const float *Wc = sW(t), *Wdn = sW(t - 1), *Gcp = sG(t), *Gup = sG(t + 1);
#pragma unroll
            for (int r = 0; r < RPW; r++) {
                u2[r] = v2[r] = w2[r] = fz[r] = zero2;
                const int Y = rowY[r], j = rowj[r];
                if (!(Y >= 2 && Y <= PH - 2)) continue;
                const bool jin = INT || (j >= 0 && j < ny);
                const bool jint = INT || (j > 0 && j < ny - 1);
                // x faces ia, ib (west faces of the pair)
                {
                    const float2 qc = ld2(Qc, Y, X), Ut = ld2(Uc, Y, X), Gt = ld2(Gcp, Y, X);
                    const float2 qcl = lft(qc), Gs = ad<EXACT>(Gt, lft(Gt));
                    float2 val;
                    if constexpr (EXACT) {
                        val = base_x(Ut, Gs, qc, qcl);
                        if (jint) {
                            const float2 qn = ld2(Qc, Y + 1, X), qs = ld2(Qc, Y - 1, X);
                            const float2 Vt = ld2(Vc, Y, X), Vtn = ld2(Vc, Y + 1, X);
                            const float2 qnl = lft(qn), qsl = lft(qs);
                            val = cross_x(val, Ut, avg4(Vt, Vtn, lft(Vt), lft(Vtn)),
                                          div2x(xnum(qn, qs, qnl, qsl), xden(qn, qs, qnl, qsl)), Gs);
                        }
                        if (kint) {
                            const float2 qu = ld2(Qu, Y, X), qd = ld2(Qd, Y, X);
                            const float2 Wt = ld2(Wc, Y, X), Wd = ld2(Wdn, Y, X);
                            const float2 qul = lft(qu), qdl = lft(qd);
                            val = cross_x(val, Ut, avg4(Wt, Wd, lft(Wt), lft(Wd)),
                                          div2x(xnum(qu, qd, qul, qdl), xden(qu, qd, qul, qdl)), Gs);
                        }
                        val = mul2x(val, splat2(0.5f));
                    } else {
                        // the final 0.5 folded in: 0.5 |U| (1 - 2 |U| / Gs) = 0.5 |U| - U^2 / Gs, and each
                        // cross term 0.25 U / Gs times the 4-face average (1/4 of the face sum) times eq
                        const float2 rG = rcp2(Gs);
                        const float2 F0 = sub2(mul2(splat2(0.5f), abs2(Ut)), mul2(mul2(Ut, Ut), rG));
                        val = mul2(mul2(F0, sub2(qc, qcl)), rcp2(add2(add2(qc, qcl), splat2(1e-10f))));
                        const float2 mc = mul2(splat2(-0.0625f), mul2(Ut, rG));
                        if (jint) {
                            const float2 qn = ld2(Qc, Y + 1, X), qs = ld2(Qc, Y - 1, X);
                            const float2 sv = add2(ld2(Vc, Y, X), ld2(Vc, Y + 1, X));
                            const float2 xp = add2(qn, lft(qn)), xm = add2(qs, lft(qs));
                            const float2 eq = mul2(sub2(xp, xm), rcp2(add2(add2(xp, xm), splat2(1e-10f))));
                            val = fma2(mul2(mc, add2(sv, lft(sv))), eq, val);
                        }
                        if (kint) {
                            const float2 qu = ld2(Qu, Y, X), qd = ld2(Qd, Y, X);
                            const float2 sw = add2(ld2(Wc, Y, X), ld2(Wdn, Y, X));
                            const float2 xp = add2(qu, lft(qu)), xm = add2(qd, lft(qd));
                            const float2 eq = mul2(sub2(xp, xm), rcp2(add2(add2(xp, xm), splat2(1e-10f))));
                            val = fma2(mul2(mc, add2(sw, lft(sw))), eq, val);
                        }
                    }
                    u2[r] = val;
                    if (!INT) {
                        u2[r].x = (jin && ia >= 1 && ia <= nx - 1) ? val.x : 0.0f;
                        u2[r].y = (jin && ib >= 1 && ib <= nx - 1) ? val.y : 0.0f;
                    }
                }
                // y face j (south faces of the pair)
                {
                    const float2 qc = ld2(Qc, Y, X), qs = ld2(Qc, Y - 1, X);
                    const float2 Vt = ld2(Vc, Y, X), Gs = ad<EXACT>(ld2(Gcp, Y, X), ld2(Gcp, Y - 1, X));
                    const float2 Ut = ld2(Uc, Y, X), Us = ld2(Uc, Y - 1, X);
                    const bool xa = INT || (ia > 0 && ia < nx - 1), xb = INT || (ib > 0 && ib < nx - 1);
                    float2 val;
                    if constexpr (EXACT) {
                        const float2 qcl = lft(qc), qcr = rgt(qc), qsl = lft(qs), qsr = rgt(qs);
                        const float2 Utr = rgt(Ut), Usr = rgt(Us);
                        val = base_x(Vt, Gs, qc, qs);
                        float2 eq = div2x(xnum(make_float2(qs.y, qsr.y), qcl, make_float2(qc.y, qcr.y), qsl),
                                          xden(make_float2(qc.y, qcr.y), make_float2(qs.y, qsr.y), qcl, qsl));
                        float2 ev = avg4(make_float2(Ut.y, Utr.y), make_float2(Us.y, Usr.y), Ut, Us);
                        if (!xa) eq.x = ev.x = 0.0f;
                        if (!xb) eq.y = ev.y = 0.0f;
                        val = cross_x(val, Vt, ev, eq, Gs);
                        if (kint) {
                            const float2 qu = ld2(Qu, Y, X), qd = ld2(Qd, Y, X);
                            const float2 qsu = ld2(Qu, Y - 1, X), qsd = ld2(Qd, Y - 1, X);
                            const float2 Wt = ld2(Wc, Y, X), Wd = ld2(Wdn, Y, X);
                            const float2 Wts = ld2(Wc, Y - 1, X), Wds = ld2(Wdn, Y - 1, X);
                            val = cross_x(val, Vt, avg4(Wt, Wd, Wts, Wds), div2x(xnum(qsu, qd, qu, qsd),
                                                                                xden(qsu, qd, qu, qsd)), Gs);
                        }
                        val = mul2x(val, splat2(0.5f));
                    } else {
                        const float2 rG = rcp2(Gs);
                        const float2 F0 = sub2(mul2(splat2(0.5f), abs2(Vt)), mul2(mul2(Vt, Vt), rG));
                        val = mul2(mul2(F0, sub2(qc, qs)), rcp2(add2(add2(qc, qs), splat2(1e-10f))));
                        const float2 mc = mul2(splat2(-0.0625f), mul2(Vt, rG));
                        // x cross term: the two rows' pair sums at x+1 and x-1, and U_m on the
                        // cells' west and east faces in both rows, each formed from one shuffle
                        const float2 sq = add2(qc, qs), yp = rgt(sq), ym = lft(sq);
                        float2 eq = mul2(sub2(yp, ym), rcp2(add2(add2(yp, ym), splat2(1e-10f))));
                        const float2 su = add2(Ut, Us);
                        float2 ev = add2(su, rgt(su));
                        // no cross term on the domain's first and last columns (their
                        // shuffled neighbours may lie outside the plane)
                        if (!xa) ev.x = eq.x = 0.0f;
                        if (!xb) ev.y = eq.y = 0.0f;
                        val = fma2(mul2(mc, ev), eq, val);
                        if (kint) {
                            const float2 zp = add2(ld2(Qu, Y, X), ld2(Qu, Y - 1, X));
                            const float2 zm = add2(ld2(Qd, Y, X), ld2(Qd, Y - 1, X));
                            const float2 eq2 = mul2(sub2(zp, zm), rcp2(add2(add2(zp, zm), splat2(1e-10f))));
                            const float2 sw = add2(add2(ld2(Wc, Y, X), ld2(Wdn, Y, X)),
                                                   add2(ld2(Wc, Y - 1, X), ld2(Wdn, Y - 1, X)));
                            val = fma2(mul2(mc, sw), eq2, val);
                        }
                    }
                    v2[r] = val;
                    if (!INT) {
                        const bool fin = j >= 1 && j <= ny - 1;
                        v2[r].x = (fin && inA) ? val.x : 0.0f;
                        v2[r].y = (fin && inB) ? val.y : 0.0f;
                    }
                    st2(P(S_V2), Y, X, v2[r]);
                }
                // z face at the top of level t (columns inside the domain interior)
                if (!top) {
                    const float2 qc = ld2(Qc, Y, X), qu = ld2(Qu, Y, X);
                    const float2 Wt = ld2(Wc, Y, X), Gs = ad<EXACT>(ld2(Gup, Y, X), ld2(Gcp, Y, X));
                    const float2 Ut = ld2(Uc, Y, X), Uu = ld2(Uup, Y, X);
                    const float2 qn = ld2(Qc, Y + 1, X), qs = ld2(Qc, Y - 1, X);
                    const float2 qnu = ld2(Qu, Y + 1, X), qsu = ld2(Qu, Y - 1, X);
                    const float2 Vt = ld2(Vc, Y, X), Vtn = ld2(Vc, Y + 1, X);
                    const float2 Vu = ld2(Vup, Y, X), Vun = ld2(Vup, Y + 1, X);
                    float2 val;
                    if constexpr (EXACT) {
                        const float2 qcl = lft(qc), qcr = rgt(qc), qul = lft(qu), qur = rgt(qu);
                        const float2 Utr = rgt(Ut), Uur = rgt(Uu);
                        val = base_x(Wt, Gs, qu, qc);
                        val = cross_x(val, Wt, avg4(make_float2(Ut.y, Utr.y), make_float2(Uu.y, Uur.y), Ut, Uu),
                                      div2x(xnum(make_float2(qu.y, qur.y), qcl, make_float2(qc.y, qcr.y), qul),
                                            xden(make_float2(qc.y, qcr.y), make_float2(qu.y, qur.y), qcl, qul)),
                                      Gs);
                        val = cross_x(val, Wt, avg4(Vt, Vu, Vtn, Vun), div2x(xnum(qnu, qs, qn, qsu), xden(qn, qsu, qnu, qs)),
                                      Gs);
                        val = mul2x(mul2x(val, splat2(0.5f)), c_dz[r]);
                    } else {
                        const float2 rG = rcp2(Gs);
                        const float2 F0 = sub2(mul2(splat2(0.5f), abs2(Wt)), mul2(mul2(Wt, Wt), rG));
                        val = mul2(mul2(F0, sub2(qu, qc)), rcp2(add2(add2(qu, qc), splat2(1e-10f))));
                        const float2 mc = mul2(splat2(-0.0625f), mul2(Wt, rG));
                        const float2 sq = add2(qc, qu), zp = rgt(sq), zm = lft(sq);
                        const float2 eq = mul2(sub2(zp, zm), rcp2(add2(add2(zp, zm), splat2(1e-10f))));
                        const float2 su = add2(Ut, Uu);
                        val = fma2(mul2(mc, add2(su, rgt(su))), eq, val);
                        const float2 np = add2(qn, qnu), sp = add2(qs, qsu);
                        const float2 eq2 = mul2(sub2(np, sp), rcp2(add2(add2(np, sp), splat2(1e-10f))));
                        const float2 sv = add2(add2(Vt, Vu), add2(Vtn, Vun));
                        val = fma2(mul2(mc, sv), eq2, val);
                        val = mul2(val, c_dz[r]);
                    }
                    w2[r] = val;
                    if (!INT) {
                        const bool jj = j >= 1 && j <= ny - 2;
                        w2[r].x = (jj && ia >= 1 && ia <= nx - 2) ? val.x : 0.0f;
                        w2[r].y = (jj && ib >= 1 && ib <= nx - 2) ? val.y : 0.0f;
                    }
                    fz[r] = flux<EXACT>(qc, qu, w2[r]);
                }
            }
            __syncthreads();   // v2 plane complete

            // ---- P2: limiter betas at level t --------------------------------
#pragma unroll
            for (int r = 0; r < RPW; r++) {
                bxi[r] = bxo[r] = byi[r] = byo[r] = bzi[r] = bzo[r] = splat2(0.0f);
                const int Y = rowY[r], j = rowj[r];
                if (!FCT || !(Y >= 2 && Y <= PH - 3)) continue;
                const float2 qc = ld2(sQ1(t), Y, X), q0c = ld2(sq0(t), Y, X);
                const float2 qcl = lft(qc), qcr = rgt(qc), q0l = lft(q0c), q0r = rgt(q0c);
                // x lines: faces ia, ib, ib+1
                {
                    const float2 fl = flux<EXACT>(qcl, qc, u2[r]), fr = rgt(fl);
                    if constexpr (INT && !EXACT) {
                        fct_pair_fast(qcl, qc, qcr, q0l, q0c, q0r, fl, fr, bxi[r], bxo[r]);
                    } else if constexpr (!EXACT) {
                        float2 a1m = qcl, a1p = qcr, a0m = q0l, a0c = q0c, a0p = q0r, afl = fl, afr = fr;
                        fct_edge_sub(ia == 0, ia == nx - 1, a1m.x, qc.x, a1p.x, a0m.x, a0c.x, a0p.x, afl.x, afr.x);
                        fct_edge_sub(ib == 0, ib == nx - 1, a1m.y, qc.y, a1p.y, a0m.y, a0c.y, a0p.y, afl.y, afr.y);
                        fct_pair_fast(a1m, qc, a1p, a0m, a0c, a0p, afl, afr, bxi[r], bxo[r]);
                    } else {
                        const int pa = INT ? 0 : (ia == 0 ? 1 : (ia == nx - 1 ? 2 : 0));
                        const int pb = INT ? 0 : (ib == 0 ? 1 : (ib == nx - 1 ? 2 : 0));
                        fct_cell<EXACT>(qcl.x, qc.x, qcr.x, q0l.x, q0c.x, q0r.x, fl.x, fr.x, pa, false, bxi[r].x,
                                        bxo[r].x);
                        fct_cell<EXACT>(qcl.y, qc.y, qcr.y, q0l.y, q0c.y, q0r.y, fl.y, fr.y, pb, false, bxi[r].y,
                                        bxo[r].y);
                    }
                }
                // y lines: faces j and j+1
                {
                    const float2 qn = ld2(sQ1(t), Y + 1, X), qs = ld2(sQ1(t), Y - 1, X);
                    const float2 q0n = ld2(sq0(t), Y + 1, X), q0s = ld2(sq0(t), Y - 1, X);
                    const float2 vn = ld2(P(S_V2), Y + 1, X);
                    const float2 fl = flux<EXACT>(qs, qc, v2[r]), fr = flux<EXACT>(qc, qn, vn);
                    if constexpr (INT && !EXACT) {
                        fct_pair_fast(qs, qc, qn, q0s, q0c, q0n, fl, fr, byi[r], byo[r]);
                    } else if constexpr (!EXACT) {
                        float2 a1m = qs, a1p = qn, a0m = q0s, a0c = q0c, a0p = q0n, afl = fl, afr = fr;
                        if (j == 0 || j == ny - 1) {   // row-uniform
                            fct_edge_sub(j == 0, j == ny - 1, a1m.x, qc.x, a1p.x, a0m.x, a0c.x, a0p.x, afl.x, afr.x);
                            fct_edge_sub(j == 0, j == ny - 1, a1m.y, qc.y, a1p.y, a0m.y, a0c.y, a0p.y, afl.y, afr.y);
                        }
                        fct_pair_fast(a1m, qc, a1p, a0m, a0c, a0p, afl, afr, byi[r], byo[r]);
                    } else {
                        const int pj = INT ? 0 : (j == 0 ? 1 : (j == ny - 1 ? 2 : 0));
                        fct_cell<EXACT>(qs.x, qc.x, qn.x, q0s.x, q0c.x, q0n.x, fl.x, fr.x, pj, false, byi[r].x,
                                        byo[r].x);
                        fct_cell<EXACT>(qs.y, qc.y, qn.y, q0s.y, q0c.y, q0n.y, fl.y, fr.y, pj, false, byi[r].y,
                                        byo[r].y);
                    }
                    st2(P(S_BYI), Y, X, byi[r]);
                    st2(P(S_BYO), Y, X, byo[r]);
                }
                // z line of the own column (fz of the faces below and above)
                {
                    const float2 qu = t < nz - 1 ? ld2(sQ1(t + 1), Y, X) : zero2;
                    const float2 qd = t > 0 ? ld2(sQ1(t - 1), Y, X) : zero2;
                    const float2 q0u = t < nz - 1 ? ld2(sq0(t + 1), Y, X) : zero2;
                    const float2 q0d = t > 0 ? ld2(sq0(t - 1), Y, X) : zero2;
                    // flux through the top of level t-1, as P1 formed it one level ago
                    const float2 fzd = flux<EXACT>(qd, qc, r_w2[r]);
                    const int pz = t == 0 ? 1 : (t == nz - 1 ? 2 : 0);
                    if (!EXACT && pz == 0) {
                        fct_pair_fast(qd, qc, qu, q0d, q0c, q0u, fzd, fz[r], bzi[r], bzo[r]);
                    } else {
                        fct_cell<EXACT>(qd.x, qc.x, qu.x, q0d.x, q0c.x, q0u.x, fzd.x, fz[r].x, pz, true, bzi[r].x,
                                        bzo[r].x);
                        fct_cell<EXACT>(qd.y, qc.y, qu.y, q0d.y, q0c.y, q0u.y, fzd.y, fz[r].y, pz, true, bzi[r].y,
                                        bzo[r].y);
                    }
                }
            }
            __syncthreads();   // y betas complete
        }

        // ---- P3: limited faces, corrective pass; output level t-1 ----------
#pragma unroll
        for (int r = 0; r < RPW; r++) {
            const int Y = rowY[r], j = rowj[r];
            const bool outrow = Y >= 3 && Y <= PH - 4;      // warp-uniform
            // n_ft: the limited flux through the top of level t-1, formed with
            // the level-t betas and carried to the next level as its bottom flux
            float2 n_part = zero2, n_ft = zero2;
            if (haveA && outrow) {
                const float2 qc = ld2(sQ1(t), Y, X), qn = ld2(sQ1(t), Y + 1, X), qs = ld2(sQ1(t), Y - 1, X);
                const float2 qcl = lft(qc);
                const float2 vn0 = ld2(P(S_V2), Y + 1, X);
                float2 fw, f3, f4;
                if constexpr (EXACT) {
                    float2 uw = u2[r], vs = v2[r], vn = vn0;
                    if (FCT) {
                        const float2 bil = lft(bxi[r]), bol = lft(bxo[r]);
                        uw.x = limit<EXACT>(uw.x, bxi[r].x, bol.x, bil.x, bxo[r].x);
                        uw.y = limit<EXACT>(uw.y, bxi[r].y, bxo[r].x, bxi[r].x, bxo[r].y);
                        const float2 bis = ld2(P(S_BYI), Y - 1, X), bos = ld2(P(S_BYO), Y - 1, X);
                        const float2 bin = ld2(P(S_BYI), Y + 1, X), bon = ld2(P(S_BYO), Y + 1, X);
                        vs.x = limit<EXACT>(vs.x, byi[r].x, bos.x, bis.x, byo[r].x);
                        vs.y = limit<EXACT>(vs.y, byi[r].y, bos.y, bis.y, byo[r].y);
                        vn.x = limit<EXACT>(vn.x, bin.x, byo[r].x, byi[r].x, bon.x);
                        vn.y = limit<EXACT>(vn.y, bin.y, byo[r].y, byi[r].y, bon.y);
                    }
                    fw = flux_x(qcl, qc, uw);
                    f3 = flux_x(qc, qn, vn);
                    f4 = flux_x(qs, qc, vs);
                } else if (FCT) {
                    const float2 bis = ld2(P(S_BYI), Y - 1, X), bos = ld2(P(S_BYO), Y - 1, X);
                    const float2 bin = ld2(P(S_BYI), Y + 1, X), bon = ld2(P(S_BYO), Y + 1, X);
                    fw = lim_flux2(u2[r], qcl, qc, bxi[r], lft(bxo[r]), lft(bxi[r]), bxo[r]);
                    f4 = lim_flux2(v2[r], qs, qc, byi[r], bos, bis, byo[r]);
                    f3 = lim_flux2(vn0, qc, qn, bin, byo[r], byi[r], bon);
                } else {
                    fw = flux_f(qcl, qc, u2[r]);
                    f3 = flux_f(qc, qn, vn0);
                    f4 = flux_f(qs, qc, v2[r]);
                }
                // east faces as the next cell's limited west faces
                const float2 fe = rgt(fw);
                const float2 hd = ad<EXACT>(sb<EXACT>(fe, fw), sb<EXACT>(f3, f4));
                const float2 G = ld2(sG(t), Y, X);
                if constexpr (EXACT) n_part = sub2x(qc, div2x(hd, G));
                else n_part = sub2(qc, mul2(hd, r_rg[r]));
                if (t >= 1) {
                    const float2 qd = ld2(sQ1(t - 1), Y, X);
                    if constexpr (EXACT) {
                        float2 w = r_w2[r];
                        if (FCT) {
                            w.x = limit<EXACT>(w.x, bzi[r].x, r_bzo[r].x, r_bzi[r].x, bzo[r].x);
                            w.y = limit<EXACT>(w.y, bzi[r].y, r_bzo[r].y, r_bzi[r].y, bzo[r].y);
                        }
                        n_ft = flux_x(qd, qc, w);
                    } else if (FCT) {
                        n_ft = lim_flux2(r_w2[r], qd, qc, bzi[r], r_bzo[r], r_bzi[r], bzo[r]);
                    } else {
                        n_ft = flux_f(qd, qc, r_w2[r]);
                    }
                }
            }
            // vertical part of level L = t-1 and the store
            if (t >= 1 && outrow) {
                const int L = t - 1;
                float2 val = r_part[r];
                const float2 djr = r_djrm[r];
                if constexpr (EXACT) {
                    if (L > 0 && L < nz - 1) {
                        val = sub2x(val, div2x(sub2x(n_ft, r_fb[r]), djr));
                    } else if (L == 0) {
                        val = sub2x(val, div2x(n_ft, djr));
                    } else {
                        // the model top: q times the (zero) face velocity there
                        const float2 qc = ld2(sQ1(L), Y, X);
                        val = sub2x(val, div2x(sub2x(mul2x(qc, zero2), r_fb[r]), djr));
                    }
                } else {
                    float2 vd;
                    if (L > 0 && L < nz - 1) vd = sub2(n_ft, r_fb[r]);
                    else if (L == 0) vd = n_ft;
                    else vd = make_float2(-r_fb[r].x, -r_fb[r].y);   // nothing leaves through the model top
                    val = sub2(val, mul2(vd, djr));
                }
                const bool jin = INT || (j >= 0 && j < ny);
                const bool jring = !INT && (j == 0 || j == ny - 1);
                const bool oa = jin && (INT || inA) && X >= xlo && X < xhi;
                const bool ob = jin && (INT || inB) && X + 1 >= xlo && X + 1 < xhi;
                float va = val.x, vb = val.y;
                if (!INT) {
                    const float2 q0L = ld2(sq0(L), Y, X);
                    va = (jring || ia == 0 || ia == nx - 1) ? q0L.x : val.x;
                    vb = (jring || ib == 0 || ib == nx - 1) ? q0L.y : val.y;
                }
                if (oa || ob) {
                    // ia is even and rows start on 16-byte boundaries: the pair is 8-byte aligned
                    float *dst = outg + ix(g, 0, L, j);
                    if (oa && ob) *reinterpret_cast<float2 *>(dst + ia) = make_float2(va, vb);
                    else if (oa) dst[ia] = va;
                    else dst[ib] = vb;
                }
            }
            // rotate the carried state
            if (haveA) {
                r_fb[r] = n_ft;
                r_part[r] = n_part;
                r_w2[r] = w2[r];
                r_bzi[r] = bzi[r];
                r_bzo[r] = bzo[r];
            }
            r_djrm[r] = r_djr0[r];
            r_djr0[r] = c_djrn[r];
        }
    }
    return true;

drain:
    // a wait gave up: wait (bounded) for both barriers' latest batches so
    // no copy is left in flight into this CTA's shared memory, then stop
    mbar_wait_bounded(&bars[0], (ph[0] - 1) & 1u, WAIT_NS);
    mbar_wait_bounded(&bars[1], (ph[1] - 1) & 1u, WAIT_NS);
    return false;
}

// Barrier set-up, once per CTA.
__device__ __forceinline__ void onepass_init_bars(uint64_t *bars, uint32_t *ph)
{
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
    }
    ph[0] = ph[1] = 0;
    __syncthreads();
}

// Whether a tile's whole plane (origin x0, first output row j0) lies inside
// the domain interior.
__device__ __forceinline__ bool onepass_interior(const Geo &g, int x0, int j0)
{
    return x0 >= 1 && x0 + op::PW - 1 <= g.nx - 2 && j0 - 3 >= 1 && j0 - 3 + op::PH - 1 <= g.ny - 2;
}

// Tile (tx, j0) of a domain: plane origin and output columns, then the march.
template <bool EXACT, bool FCT>
__device__ __forceinline__ bool onepass_run(float *sm, uint64_t *bars, uint32_t *ph, const OnePassParams &p, int s,
                                            int tx, int j0)
{
    int x0, xlo, xhi;
    op::xtile(p.g.nx, tx, p.tiles_x, x0, xlo, xhi);
    if (onepass_interior(p.g, x0, j0)) return onepass_tile<EXACT, FCT, true>(sm, bars, ph, p, s, x0, xlo, xhi, j0);
    return onepass_tile<EXACT, FCT, false>(sm, bars, ph, p, s, x0, xlo, xhi, j0);
}

template <bool EXACT, bool FCT>
__global__ void __launch_bounds__(op::NT, 1) k_mpdata_onepass(const __grid_constant__ OnePassParams p)
{
    using namespace op;
    extern __shared__ float4 smem4[];
    // planes start on 128-byte boundaries (TMA destinations); SMEM has the slack
    float *sm = reinterpret_cast<float *>(smem4) + ((128u - (smem_u32(smem4) & 127u)) & 127u) / sizeof(float);
    __shared__ __align__(8) uint64_t bars[2];
    const int s = blockIdx.x % p.nspecies;
    const int tile = blockIdx.x / p.nspecies;
    const int tx = tile % p.tiles_x, j0 = (tile / p.tiles_x) * TY;
    __shared__ int stop;
    if (threadIdx.x == 0) stop = *reinterpret_cast<volatile const int *>(p.err);
    __syncthreads();
    if (stop) return;   // an earlier tile of this launch gave up on a TMA wait: stop (the whole CTA)
    uint32_t ph[2];
    onepass_init_bars(bars, ph);
    onepass_run<EXACT, FCT>(sm, bars, ph, p, s, tx, j0);
}

// Batched form: one launch over the work list of (member, species, column
// tile tx, first row j0) items, one CTA per item; params[member] holds that
// member's descriptors, pointers and geometry for the current buffer
// parity.  The hardware block scheduler hands out the items in list order
// as SMs free up.  (A persistent form, CTAs pulling items with an atomic
// counter, carried its barrier phases and item bookkeeping through the
// march, spilled some 400 bytes per thread to local memory and ran the
// 64-member ensemble 1.5x slower.)
template <bool EXACT, bool FCT>
__global__ void __launch_bounds__(op::NT, 1)
    k_batch_onepass_items(const OnePassParams *__restrict__ params, const int4 *__restrict__ items)
{
    extern __shared__ float4 smem4[];
    float *sm = reinterpret_cast<float *>(smem4) + ((128u - (smem_u32(smem4) & 127u)) & 127u) / sizeof(float);
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ __align__(16) OnePassParams sp;
    __shared__ int stop;
    constexpr int PW4 = (int)(sizeof(OnePassParams) / sizeof(int));
    const int4 w = items[blockIdx.x];
    const int *src = reinterpret_cast<const int *>(params + w.x);
    for (int q = threadIdx.x; q < PW4; q += blockDim.x) reinterpret_cast<int *>(&sp)[q] = src[q];
    // an earlier tile of this launch gave up on a TMA wait: stop (the whole CTA)
    if (threadIdx.x == 0) stop = *reinterpret_cast<volatile const int *>(params[0].err);
    __syncthreads();
    if (stop) return;
    uint32_t ph[2];
    onepass_init_bars(bars, ph);
    onepass_run<EXACT, FCT>(sm, bars, ph, sp, w.y, w.z, w.w);
}

}  // namespace icar
