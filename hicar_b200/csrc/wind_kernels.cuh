// Wind balance and the stable time step on the device: the two per-step
// wind operations that sit next to advection in ICAR's time loop.
//
//   k_balance_uvw   balance_uvw (src/physics/wind.f90:88-164) with
//                   calc_divergence(horz_only) and calc_w (:166-271): one
//                   thread per (i, j) column marches up the column, forming
//                   the horizontal divergence of the metric-weighted u, v at
//                   each level and integrating w from w = 0 below the ground;
//                   the levels arrive in shared-memory planes ahead of use.
//   k_dt_maxima     the maxima compute_dt (src/main/time_step.f90:51-168)
//                   needs: max |u|, |v|, |w| over the whole arrays and the
//                   per-cell CFL rate max(|u|/dx, |v|/dx, |w|/dz) over the
//                   tile, reduced in the block and combined with atomicMax
//                   on the bit patterns (order-preserving for values >= 0).
//
// Both are single passes over the fields (HBM bound); the expressions keep
// the Fortran evaluation order, like the advection kernels.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"
#include "mpdata_fused.cuh"

namespace icar {

namespace balf {
// CTA tile: 32 x 8 columns, one thread per column marching up k.  The
// seven fields a level needs (u, J_u, v, J_v, rho, dz, J_w) arrive in
// shared-memory planes by 16-byte cp.async, DEPTH levels ahead of use:
// each plane spans x from i0-4 (a multiple of 4) to i0+35 and y from j0-1
// to j0+8, covering the faces i0..i0+32 / j0..j0+8 and the density
// neighbours the face weights read.
constexpr int BX = 32, BY = 8, NT = BX * BY;
constexpr int PW = 40, PH = BY + 2, PLANE = PW * PH;
constexpr int NF = 7;                      // u, ju, v, jv, rho, dz, jw
constexpr int DEPTH = 3, NSLOT = DEPTH + 1;
constexpr int CPR = PW / 4, NCH = (NF * CPR * PH + NT - 1) / NT;
constexpr size_t SMEM = (size_t)NSLOT * NF * PLANE * sizeof(float);
}  // namespace balf

// u*J_u on x face f, times the face density when advect_density (the
// outermost faces extrapolate it), wind.f90:237-239.  U, JU, R point at
// the cell's row of the u, J_u and density planes; plane column = index -
// ox.
__device__ __forceinline__ float umet_p(int nx, int adv_den, const float *U, const float *JU, const float *R, int f,
                                        int ox)
{
    const int p = f - ox;
    const float uj = U[p] * JU[p];
    if (!adv_den) return uj;
    if (f == 0) return uj * (1.5f * R[0 - ox] - 0.5f * R[1 - ox]);
    if (f == nx) return uj * (1.5f * R[nx - 1 - ox] - 0.5f * R[nx - 2 - ox]);
    return uj * (R[p - 1] + R[p]) / 2.0f;
}

// v*J_v on y face gy, wind.f90:241-243; V, JV, R point at row gy of the v,
// J_v and density planes in the cell's column (rows of stride balf::PW).
__device__ __forceinline__ float vmet_p(int ny, int adv_den, const float *V, const float *JV, const float *R, int gy)
{
    constexpr int W = balf::PW;
    const float vj = V[0] * JV[0];
    if (!adv_den) return vj;
    if (gy == 0) return vj * (1.5f * R[0] - 0.5f * R[W]);
    if (gy == ny) return vj * (1.5f * R[-W] - 0.5f * R[-2 * W]);
    return vj * (R[-W] + R[0]) / 2.0f;
}

// Columns i_s..i_e x j_s..j_e (its-1..ite+1 clipped to the domain, i.e.
// [max(hs-1,0), min(n-hs,n-1)] for one image with halo hs) get the balanced
// w; every other column gets w = 0 (calc_w sets the whole array first).
__global__ void __launch_bounds__(balf::NT)
    k_balance_uvw(Geo g, int hs, float dx, int adv_den, const float *__restrict__ u, const float *__restrict__ v,
                  const float *__restrict__ rho, const float *__restrict__ dz, const float *__restrict__ ju,
                  const float *__restrict__ jv, const float *__restrict__ jw, float *__restrict__ w)
{
    using namespace balf;
    extern __shared__ float4 sm4[];
    float *sm = reinterpret_cast<float *>(sm4);
    const int tx = threadIdx.x % BX, ty = threadIdx.x / BX;
    const int i0 = blockIdx.x * BX, j0 = blockIdx.y * BY;
    const int i = i0 + tx, j = j0 + ty;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int ox = i0 - 4, oy = j0 - 1;
    const int i_s = max(hs - 1, 0), i_e = min(nx - hs, nx - 1);
    const int j_s = max(hs - 1, 0), j_e = min(ny - hs, ny - 1);
    const bool in = i < nx && j < ny;
    const bool bal = in && i >= i_s && i <= i_e && j >= j_s && j <= j_e;
    // every thread's chunks of one level: field f, row ly, chunk cx
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
        src[c] = u;
        if (e < NF * CPR * PH) {
            const int f = e / (CPR * PH), r = e % (CPR * PH);
            const int ly = r / CPR, cx = r % CPR;
            const int gi = ox + 4 * cx, gj = oy + ly;
            const bool yface = f == 2 || f == 3;
            dst[c] = f * PLANE + ly * PW + 4 * cx;
            src[c] = f == 0 ? u : f == 1 ? ju : f == 2 ? v : f == 3 ? jv : f == 4 ? rho : f == 5 ? dz : jw;
            ok[c] = gi >= 0 && gi < g.P && gj >= 0 && gj < (yface ? ny + 1 : ny);
            if (ok[c]) off[c] = (size_t)gi + (size_t)g.P * nz * gj;
        }
    }
    auto issue = [&](int k) {
        if (k < nz) {
            float *slot = sm + (size_t)(k % NSLOT) * NF * PLANE;
            const size_t lo = (size_t)k * g.P;
#pragma unroll
            for (int c = 0; c < NCH; c++)
                if (dst[c] >= 0) cp_async16(slot + dst[c], ok[c] ? src[c] + off[c] + lo : src[c], ok[c]);
        }
        cp_async_commit();
    };
#pragma unroll
    for (int k = 0; k < DEPTH; k++) issue(k);
    float wb = 0.0f, rib = 0.0f, jwb = 0.0f;  // w, interface density and J_w one level down
    const int px = i - ox, py = j - oy;
    for (int k = 0; k < nz; k++) {
        cp_async_wait<DEPTH - 2>();  // levels k and k+1 have landed
        __syncthreads();
        issue(k + DEPTH);            // into the slot of level k-1, read by nobody any more
        const float *L = sm + (size_t)(k % NSLOT) * NF * PLANE;
        const float *Lu = sm + (size_t)((k + 1) % NSLOT) * NF * PLANE;
        const size_t c = ix(g, i, k, j);
        if (!bal) {
            if (in) w[c] = 0.0f;
            continue;
        }
        const float *U = L, *JU = L + PLANE, *V = L + 2 * PLANE, *JV = L + 3 * PLANE, *R = L + 4 * PLANE;
        const float *DZ = L + 5 * PLANE, *JW = L + 6 * PLANE;
        const float *Ur = U + py * PW, *JUr = JU + py * PW, *Rr = R + py * PW;
        const float ue = umet_p(nx, adv_den, Ur, JUr, Rr, i + 1, ox), uw = umet_p(nx, adv_den, Ur, JUr, Rr, i, ox);
        const int pc = py * PW + px;
        const float vn = vmet_p(ny, adv_den, V + pc + PW, JV + pc + PW, R + pc + PW, j + 1);
        const float vs = vmet_p(ny, adv_den, V + pc, JV + pc, R + pc, j);
        const float div = ((ue - uw) + (vn - vs)) / dx;
        const float d = DZ[pc], jwc = JW[pc];
        float wk;
        if (adv_den) {
            // rho_i(k) = (rho_k*dz_k + rho_k+1*dz_k+1) / (dz_k + dz_k+1), wind.f90:175-176
            float ri = 0.0f;
            if (k < nz - 1) {
                const float dzu = Lu[5 * PLANE + pc];
                ri = (R[pc] * d + Lu[4 * PLANE + pc] * dzu) / (d + dzu);
            }
            if (k == 0)
                wk = 0.0f - div * d / (jwc * ri);
            else if (k == nz - 1)
                wk = ((wb * rib * jwb) - div * d) / (jwc * R[pc]);
            else
                wk = ((wb * rib * jwb) - div * d) / (jwc * ri);
            rib = ri;
        } else {
            if (k == 0)
                wk = (0.0f - div * d) / jwc;
            else
                wk = (wb * jwb - div * d) / jwc;
        }
        w[c] = wk;
        wb = wk;
        jwb = jwc;
    }
    cp_async_wait<0>();
}

// out[0..2] = bits of max |u|, |v|, |w| over the arrays; out[3] = bits of
// the largest per-cell rate over the tile (i, j in [hs, n-1-hs], every k).
// out must be zero on entry.  dzl is dz_levels (nz).
__global__ void k_dt_maxima(Geo g, int hs, float dx, const float *__restrict__ u, const float *__restrict__ v,
                            const float *__restrict__ w, const float *__restrict__ dzl, unsigned *__restrict__ out)
{
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    float mu = 0.0f, mv = 0.0f, mw = 0.0f, m3 = 0.0f;
    const size_t total = (size_t)(nx + 1) * nz * (ny + 1);  // covers u (nx+1 wide) and v (ny+1 rows)
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(t % (size_t)(nx + 1));
        const size_t rest = t / (size_t)(nx + 1);
        const int k = (int)(rest % (size_t)nz);
        const int j = (int)(rest / (size_t)nz);
        const size_t c = ix(g, i, k, j);
        if (j < ny) mu = fmax_(mu, fabsf(u[c]));
        if (i < nx) mv = fmax_(mv, fabsf(v[c]));
        if (i < nx && j < ny) mw = fmax_(mw, fabsf(w[c]));
        if (i >= hs && i <= nx - 1 - hs && j >= hs && j <= ny - 1 - hs) {
            const size_t cb = k == 0 ? c : c - (size_t)g.P;
            const float cu = fmax_(fabsf(u[c]), fabsf(u[c + 1])) / dx;
            const float cv = fmax_(fabsf(v[c]), fabsf(v[c + (size_t)g.P * nz])) / dx;
            const float cw = fmax_(fabsf(w[c]), fabsf(w[cb])) / dzl[k];
            m3 = fmax_(m3, fmax_(fmax_(cu, cv), cw));
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        mu = fmax_(mu, __shfl_xor_sync(0xffffffffu, mu, o));
        mv = fmax_(mv, __shfl_xor_sync(0xffffffffu, mv, o));
        mw = fmax_(mw, __shfl_xor_sync(0xffffffffu, mw, o));
        m3 = fmax_(m3, __shfl_xor_sync(0xffffffffu, m3, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&out[0], __float_as_uint(mu));
        atomicMax(&out[1], __float_as_uint(mv));
        atomicMax(&out[2], __float_as_uint(mw));
        atomicMax(&out[3], __float_as_uint(m3));
    }
}

// compute_dt's combination of the maxima for cfl_strictness 1..5 (host
// side, same FP32 operations as the reference).  use_density: the
// reference's density-weighted terms are commented out, so the winds then
// contribute nothing and dt is infinite.
inline float dt_from_maxima(const float m[4], float cfl, int strictness, int use_density)
{
    const float three_d_cfl = 0.577350269f;
    const float sqrt3 = std::sqrt(3.0f) * 1.001f;
    float maxwind1d = 0.0f, maxwind3d = 0.0f;
    auto mx = [](float a, float b) { return a > b ? a : b; };
    if (strictness == 1) {
        if (!use_density) maxwind1d = mx(mx(m[0], m[1]), m[2]);
        maxwind3d = maxwind1d * sqrt3;
    } else if (strictness == 5) {
        if (!use_density) maxwind3d = m[0] + m[1] + m[2];
    } else {
        if (!use_density) maxwind3d = m[3];
        if (strictness == 2) {
            maxwind3d = maxwind3d * three_d_cfl;
            if (!use_density) maxwind1d = mx(mx(m[0], m[1]), m[2]);
            maxwind3d = mx(maxwind1d, maxwind3d);
        } else if (strictness == 4) {
            maxwind3d = maxwind3d * sqrt3;
        }
    }
    return cfl / maxwind3d;
}

}  // namespace icar
