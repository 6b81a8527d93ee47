// Wind balance and the stable time step on the device: the two per-step
// wind operations that sit next to advection in ICAR's time loop.
//
//   k_balance_uvw   balance_uvw (src/physics/wind.f90:88-164) with
//                   calc_divergence(horz_only) and calc_w (:166-271): one
//                   thread per (i, j) column marches up the column, forming
//                   the horizontal divergence of the metric-weighted u, v at
//                   each level and integrating w from w = 0 below the ground.
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

namespace icar {

// u*J_u on x face f, times the face density when advect_density (the
// outermost faces extrapolate it), wind.f90:237-239.
__device__ __forceinline__ float umet(const Geo &g, int adv_den, const float *__restrict__ u,
                                      const float *__restrict__ ju, const float *__restrict__ rho, int f, int k, int j)
{
    const size_t c = ix(g, f, k, j);
    const float uj = u[c] * ju[c];
    if (!adv_den) return uj;
    if (f == 0) return uj * (1.5f * rho[ix(g, 0, k, j)] - 0.5f * rho[ix(g, 1, k, j)]);
    if (f == g.nx) return uj * (1.5f * rho[ix(g, g.nx - 1, k, j)] - 0.5f * rho[ix(g, g.nx - 2, k, j)]);
    return uj * (rho[c - 1] + rho[c]) / 2.0f;
}

// v*J_v on y face gy, wind.f90:241-243.
__device__ __forceinline__ float vmet(const Geo &g, int adv_den, const float *__restrict__ v,
                                      const float *__restrict__ jv, const float *__restrict__ rho, int i, int k, int gy)
{
    const size_t c = ix(g, i, k, gy);
    const float vj = v[c] * jv[c];
    if (!adv_den) return vj;
    if (gy == 0) return vj * (1.5f * rho[ix(g, i, k, 0)] - 0.5f * rho[ix(g, i, k, 1)]);
    if (gy == g.ny) return vj * (1.5f * rho[ix(g, i, k, g.ny - 1)] - 0.5f * rho[ix(g, i, k, g.ny - 2)]);
    return vj * (rho[ix(g, i, k, gy - 1)] + rho[c]) / 2.0f;
}

// Columns i_s..i_e x j_s..j_e (its-1..ite+1 clipped to the domain, i.e.
// [max(hs-1,0), min(n-hs,n-1)] for one image with halo hs) get the balanced
// w; every other column gets w = 0 (calc_w sets the whole array first).
__global__ void k_balance_uvw(Geo g, int hs, float dx, int adv_den, const float *__restrict__ u,
                              const float *__restrict__ v, const float *__restrict__ rho,
                              const float *__restrict__ dz, const float *__restrict__ ju,
                              const float *__restrict__ jv, const float *__restrict__ jw, float *__restrict__ w)
{
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(t % (size_t)g.nx);
    const int j = (int)(t / (size_t)g.nx);
    if (j >= g.ny) return;
    const int i_s = max(hs - 1, 0), i_e = min(g.nx - hs, g.nx - 1);
    const int j_s = max(hs - 1, 0), j_e = min(g.ny - hs, g.ny - 1);
    const int nz = g.nz;
    if (i < i_s || i > i_e || j < j_s || j > j_e) {
        for (int k = 0; k < nz; k++) w[ix(g, i, k, j)] = 0.0f;
        return;
    }
    float wb = 0.0f, rib = 0.0f;  // w and the interface density one level down
    for (int k = 0; k < nz; k++) {
        const size_t c = ix(g, i, k, j);
        const float ue = umet(g, adv_den, u, ju, rho, i + 1, k, j), uw = umet(g, adv_den, u, ju, rho, i, k, j);
        const float vn = vmet(g, adv_den, v, jv, rho, i, k, j + 1), vs = vmet(g, adv_den, v, jv, rho, i, k, j);
        const float div = ((ue - uw) + (vn - vs)) / dx;
        const float d = dz[c], jwc = jw[c];
        float wk;
        if (adv_den) {
            // rho_i(k) = (rho_k*dz_k + rho_k+1*dz_k+1) / (dz_k + dz_k+1), wind.f90:175-176
            float ri = 0.0f;
            if (k < nz - 1) {
                const size_t cu = c + (size_t)g.P;
                ri = (rho[c] * d + rho[cu] * dz[cu]) / (d + dz[cu]);
            }
            if (k == 0)
                wk = 0.0f - div * d / (jwc * ri);
            else if (k == nz - 1)
                wk = ((wb * rib * jw[c - (size_t)g.P]) - div * d) / (jwc * rho[c]);
            else
                wk = ((wb * rib * jw[c - (size_t)g.P]) - div * d) / (jwc * ri);
            rib = ri;
        } else {
            if (k == 0)
                wk = (0.0f - div * d) / jwc;
            else
                wk = (wb * jw[c - (size_t)g.P] - div * d) / jwc;
        }
        w[c] = wk;
        wb = wk;
    }
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
