// Standard (kADV_STD) advection kernels, one stage per kernel.
//   k_std_wind         adv_std_compute_wind   src/physics/advect.f90:447-493
//   k_flux3            flux3                  src/physics/advect.f90:134-251
//   k_std_update       adv_std_advect3d update src/physics/advect.f90:298-309
//   k_upflux_*         upwind_flux3           src/physics/adv_fluxcorr.f90:144-192
//   k_wrf_*            WRF_flux_corr          src/physics/adv_fluxcorr.f90:37-142
// z fluxes use an (nz+1)-level layout: level k is the bottom face of cell k,
// level 0 the ground (always 0) and level nz the model top.
#pragma once
#include "common.cuh"
#include "const_div.h"

namespace icar {

// x/12 and x/60 of the flux formulas, correctly rounded, as one double
// product (const_div.h): branch-free, unlike the general division.
__device__ __forceinline__ float div12(float x) { return __double2float_rn(__dmul_rn((double)x, ICAR_RCP12_D)); }
__device__ __forceinline__ float div60(float x) { return __double2float_rn(__dmul_rn((double)x, ICAR_RCP60_D)); }

__device__ __forceinline__ size_t izf(const Geo &g, int i, int k, int j)
{
    return (size_t)i + (size_t)g.P * ((size_t)k + (size_t)(g.nz + 1) * (size_t)j);
}

struct Idx3s {
    int i, k, j;
    bool ok;
};
__device__ __forceinline__ Idx3s decode_s(int ni, int nk, int nj)
{
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    Idx3s r;
    r.i = (int)(t % (size_t)ni);
    size_t rest = t / (size_t)ni;
    r.k = (int)(rest % (size_t)nk);
    r.j = (int)(rest / (size_t)nk);
    r.ok = r.j < nj;
    return r;
}

__global__ void k_std_wind(Geo g, float dx, float dt, int adv_den, const float *__restrict__ u,
                           const float *__restrict__ v, const float *__restrict__ w,
                           const float *__restrict__ rho, const float *__restrict__ ju,
                           const float *__restrict__ jv, const float *__restrict__ jw,
                           const float *__restrict__ dz, float *__restrict__ Um, float *__restrict__ Vm,
                           float *__restrict__ Wm)
{
    Idx3s t = decode_s(g.nx + 1, g.nz, g.ny + 1);
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
                size_t c1 = ix(g, i, k + 1, j);
                float r1 = adv_den ? rho[c1] : 1.0f;
                float d0 = dz[c], d1 = dz[c1];
                float rho_i = (r0 * d0 + r1 * d1) / (d0 + d1);
                Wm[c] = w[c] * dt * jw[c] * rho_i;
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

// Horizontal flux of order 1/3/5 across the face between r[-1] and r[0];
// r points at the cell right of (or north of) the face, s is the element
// stride along the flux direction.
__device__ __forceinline__ float hflux(int hord, const float *r, size_t s, float uu)
{
#define R(d) r[(ptrdiff_t)(d) * (ptrdiff_t)s]
    float F;
    if (hord == 1) {
        F = flux1(R(-1), R(0), uu);
    } else if (hord == 3) {
        F = 7.0f * (R(0) + R(-1)) - (R(1) + R(-2));
        F = div12(uu * F);
        F = F - div12(fabsf(uu)) * (3.0f * (R(0) - R(-1)) - (R(1) - R(-2)));
    } else {
        F = 37.0f * (R(0) + R(-1)) - 8.0f * (R(1) + R(-2)) + (R(2) + R(-3));
        F = div60(uu * F);
        F = F - div60(fabsf(uu)) * (10.0f * (R(0) - R(-1)) - 5.0f * (R(1) - R(-2)) + (R(2) - R(-3)));
    }
#undef R
    return F;
}

// flux3 over the flux region [is,ie]x[js,je] with Courant fluxes scaled by
// t_factor.  Threads cover i in [0,nx], k in [0,nz], j in [0,ny].
__global__ void k_flux3(Geo g, int hord, int vord, int is, int ie, int js, int je, float t_factor,
                        const float *__restrict__ q, const float *__restrict__ Um,
                        const float *__restrict__ Vm, const float *__restrict__ Wm,
                        float *__restrict__ fx, float *__restrict__ fy, float *__restrict__ fz)
{
    Idx3s t = decode_s(g.nx + 1, g.nz + 1, g.ny + 1);
    if (!t.ok) return;
    const int i = t.i, k = t.k, j = t.j, nz = g.nz;
    const size_t sy = (size_t)g.P * g.nz, sz = (size_t)g.P;
    if (k < nz) {
        if (j >= js && j <= je && i >= is && i <= ie + 1) {
            size_t c = ix(g, i, k, j);
            fx[c] = hflux(hord, q + c, 1, Um[c] * t_factor);
        }
        if (i >= is && i <= ie && j >= js && j <= je + 1) {
            size_t c = ix(g, i, k, j);
            fy[c] = hflux(hord, q + c, sy, Vm[c] * t_factor);
        }
    }
    if (i >= is && i <= ie && j >= js && j <= je) {
        size_t zf = izf(g, i, k, j);
        const float *col = q + ix(g, i, 0, j);
        const float *wc = Wm + ix(g, i, 0, j);
#define QZ(kk) col[(size_t)(kk) * sz]
        if (k == 0) {
            fz[zf] = 0.0f;
        } else if (k == nz) {
            fz[zf] = QZ(nz - 1) * (wc[(size_t)(nz - 1) * sz] * t_factor);
        } else {
            float ww = wc[(size_t)(k - 1) * sz] * t_factor, F;
            bool hi = (vord == 3 || vord == 5) && k >= 2 && k <= nz - 2;
            if (vord == 1 || !hi) {
                F = flux1(QZ(k - 1), QZ(k), ww);
            } else if (vord == 3 || k == 2 || k == nz - 2) {
                F = 7.0f * (QZ(k) + QZ(k - 1)) - (QZ(k + 1) + QZ(k - 2));
                F = div12(ww * F);
                F = F - div12(fabsf(ww)) * (3.0f * (QZ(k) - QZ(k - 1)) - (QZ(k + 1) - QZ(k - 2)));
            } else {
                F = 37.0f * (QZ(k) + QZ(k - 1)) - 8.0f * (QZ(k + 1) + QZ(k - 2)) + (QZ(k + 2) + QZ(k - 3));
                F = div60(ww * F);
                F = F - div60(fabsf(ww)) *
                            (10.0f * (QZ(k) - QZ(k - 1)) - 5.0f * (QZ(k + 1) - QZ(k - 2)) + (QZ(k + 2) - QZ(k - 3)));
            }
            fz[zf] = F;
        }
#undef QZ
    }
}

// qout = qold, then the flux divergence on the tile [its,ite]x[jts,jte].
// Safe in place (qout == qold): each thread reads and writes its own cell.
__global__ void k_std_update(Geo g, int its, int ite, int jts, int jte, const float *__restrict__ qold,
                             const float *__restrict__ fx, const float *__restrict__ fy,
                             const float *__restrict__ fz, const float *__restrict__ jaco,
                             const float *__restrict__ rho, int adv_den, const float *__restrict__ dz,
                             float *qout)
{
    Idx3s t = decode_s(g.nx, g.nz, g.ny);
    if (!t.ok) return;
    const int i = t.i, k = t.k, j = t.j;
    const size_t c = ix(g, i, k, j);
    float q = qold[c];
    if (i >= its && i <= ite && j >= jts && j <= jte) {
        const size_t sy = (size_t)g.P * g.nz;
        float r = adv_den ? rho[c] : 1.0f;
        float tq = q - ((fx[c + 1] - fx[c]) + (fy[c + sy] - fy[c])) / (jaco[c] * r);
        q = tq - (fz[izf(g, i, k + 1, j)] - fz[izf(g, i, k, j)]) / (dz[c] * jaco[c] * r);
    }
    qout[c] = q;
}

// ---- WRF monotonic flux correction ----------------------------------------
// Half-step upwind flux 0.5*((U+|U|)*l + (U-|U|)*r)/2, adv_fluxcorr.f90:163-168.
__device__ __forceinline__ float half_up(float U, float l, float r)
{
    float a = fabsf(U);
    return (0.5f * ((U + a) * l + (U - a) * r)) / 2.0f;
}

// pass 0: upwind fluxes of q; pass 1: add the fluxes of the predictor dq.
// Region [is,ie]x[js,je] is the tile extended by one cell.
__global__ void k_upflux(Geo g, int pass, int is, int ie, int js, int je, const float *__restrict__ s,
                         const float *__restrict__ Um, const float *__restrict__ Vm,
                         const float *__restrict__ Wm, float *__restrict__ ufx, float *__restrict__ ufy,
                         float *__restrict__ ufz)
{
    Idx3s t = decode_s(g.nx + 1, g.nz + 1, g.ny + 1);
    if (!t.ok) return;
    const int i = t.i, k = t.k, j = t.j, nz = g.nz;
    const size_t sy = (size_t)g.P * g.nz, sz = (size_t)g.P;
    if (k < nz) {
        if (j >= js && j <= je && i >= is && i <= ie + 1) {
            size_t c = ix(g, i, k, j);
            float F = half_up(Um[c], s[c - 1], s[c]);
            ufx[c] = pass == 0 ? F : ufx[c] + F;
        }
        if (i >= is && i <= ie && j >= js && j <= je + 1) {
            size_t c = ix(g, i, k, j);
            float F = half_up(Vm[c], s[c - sy], s[c]);
            ufy[c] = pass == 0 ? F : ufy[c] + F;
        }
    }
    if (i >= is && i <= ie && j >= js && j <= je) {
        size_t zf = izf(g, i, k, j);
        size_t c0 = ix(g, i, 0, j);
        if (k == 0) {
            if (pass == 0) ufz[zf] = 0.0f;
        } else if (k == nz) {
            float F = 0.5f * s[c0 + (size_t)(nz - 1) * sz] * Wm[c0 + (size_t)(nz - 1) * sz];
            ufz[zf] = pass == 0 ? F : ufz[zf] + F;
        } else {
            float F = half_up(Wm[c0 + (size_t)(k - 1) * sz], s[c0 + (size_t)(k - 1) * sz], s[c0 + (size_t)k * sz]);
            ufz[zf] = pass == 0 ? F : ufz[zf] + F;
        }
    }
}

// dq = q - div(upwind fluxes) on the extended tile; dq = q elsewhere.
__global__ void k_upflux_predict(Geo g, int is, int ie, int js, int je, const float *__restrict__ q,
                                 const float *__restrict__ ufx, const float *__restrict__ ufy,
                                 const float *__restrict__ ufz, const float *__restrict__ jaco,
                                 const float *__restrict__ rho, int adv_den, const float *__restrict__ dz,
                                 float *__restrict__ dq)
{
    Idx3s t = decode_s(g.nx, g.nz, g.ny);
    if (!t.ok) return;
    const int i = t.i, k = t.k, j = t.j;
    const size_t c = ix(g, i, k, j), sy = (size_t)g.P * g.nz;
    float v = q[c];
    if (i >= is && i <= ie && j >= js && j <= je) {
        float r = adv_den ? rho[c] : 1.0f;
        float tq = v - ((ufx[c + 1] - ufx[c]) + (ufy[c + sy] - ufy[c])) / (jaco[c] * r);
        v = tq - (ufz[izf(g, i, k + 1, j)] - ufz[izf(g, i, k, j)]) / (dz[c] * jaco[c] * r);
    }
    dq[c] = v;
}

// merged flux = high-order flux - upwind flux, over the extended face sets.
__global__ void k_wrf_merge(Geo g, int is, int ie, int js, int je, float *__restrict__ fx,
                            float *__restrict__ fy, float *__restrict__ fz, const float *__restrict__ ufx,
                            const float *__restrict__ ufy, const float *__restrict__ ufz)
{
    Idx3s t = decode_s(g.nx + 1, g.nz + 1, g.ny + 1);
    if (!t.ok) return;
    const int i = t.i, k = t.k, j = t.j;
    if (k < g.nz) {
        if (j >= js && j <= je && i >= is && i <= ie + 1) {
            size_t c = ix(g, i, k, j);
            fx[c] = fx[c] - ufx[c];
        }
        if (i >= is && i <= ie && j >= js && j <= je + 1) {
            size_t c = ix(g, i, k, j);
            fy[c] = fy[c] - ufy[c];
        }
    }
    if (i >= is && i <= ie && j >= js && j <= je) {
        size_t zf = izf(g, i, k, j);
        fz[zf] = fz[zf] - ufz[zf];
    }
}

// Per cell of the extended tile: upwind-only value, in/out flux sums,
// upwind-direction bounds and the two scale factors (adv_fluxcorr.f90:66-115).
__global__ void k_wrf_cells(Geo g, int is, int ie, int js, int je, const float *__restrict__ q,
                            const float *__restrict__ Um, const float *__restrict__ Vm,
                            const float *__restrict__ Wm, const float *__restrict__ fx,
                            const float *__restrict__ fy, const float *__restrict__ fz,
                            const float *__restrict__ ufx, const float *__restrict__ ufy,
                            const float *__restrict__ ufz, const float *__restrict__ jaco,
                            const float *__restrict__ rho, int adv_den, const float *__restrict__ dz,
                            float *__restrict__ sin_, float *__restrict__ sout)
{
    Idx3s t = decode_s(g.nx, g.nz, g.ny);
    if (!t.ok) return;
    const int i = t.i, k = t.k, j = t.j, nz = g.nz;
    if (!(i >= is && i <= ie && j >= js && j <= je)) return;
    const size_t c = ix(g, i, k, j), sy = (size_t)g.P * g.nz, sz = (size_t)g.P;
    const float e15 = 1e-15f;
    float r = adv_den ? rho[c] : 1.0f;
    float jr = jaco[c] * r, djr = dz[c] * jaco[c] * r;
    const size_t zt = izf(g, i, k + 1, j), zb = izf(g, i, k, j);
    float tq = q[c] - ((ufx[c + 1] - ufx[c]) + (ufy[c + sy] - ufy[c])) / jr;
    float temp = tq - (ufz[zt] - ufz[zb]) / djr;
    float xr = fx[c + 1], xl = fx[c], yr = fy[c + sy], yl = fy[c], ztp = fz[zt], zbt = fz[zb];
    float a = -(((fmin_(0.0f, xr) - fmax_(0.0f, xl)) + (fmin_(0.0f, yr) - fmax_(0.0f, yl))) / jr);
    float fin = a - (fmin_(0.0f, ztp) - fmax_(0.0f, zbt)) / djr;
    float b = ((fmax_(0.0f, xr) - fmin_(0.0f, xl)) + (fmax_(0.0f, yr) - fmin_(0.0f, yl))) / jr;
    float fout = b + (fmax_(0.0f, ztp) - fmin_(0.0f, zbt)) / djr;
    float mx = q[c], mn = q[c];
    if (Um[c] > 0.0f) {
        mx = fmax_(q[c - 1], mx);
        mn = fmin_(q[c - 1], mn);
    } else if (Um[c + 1] < 0.0f) {
        mx = fmax_(q[c + 1], mx);
        mn = fmin_(q[c + 1], mn);
    }
    if (Vm[c] > 0.0f) {
        mx = fmax_(q[c - sy], mx);
        mn = fmin_(q[c - sy], mn);
    } else if (Vm[c + sy] < 0.0f) {
        mx = fmax_(q[c + sy], mx);
        mn = fmin_(q[c + sy], mn);
    }
    if (k > 0 && Wm[c - sz] > 0.0f) {
        mx = fmax_(q[c - sz], mx);
        mn = fmin_(q[c - sz], mn);
    }
    if (k < nz - 1 && Wm[c] < 0.0f) {
        mx = fmax_(q[c + sz], mx);
        mn = fmin_(q[c + sz], mn);
    }
    float si = 1.0f, so = 1.0f;
    if (fin > (mx - temp)) si = fmax_(0.0f, (mx - temp) / (fin + e15));
    if (fout > (temp - mn)) so = fmax_(0.0f, (temp - mn) / (fout + e15));
    sin_[c] = si;
    sout[c] = so;
}

// Scale the interior faces and add the upwind fluxes back (:119-140).
__global__ void k_wrf_scale(Geo g, int its, int ite, int jts, int jte, float *__restrict__ fx,
                            float *__restrict__ fy, float *__restrict__ fz, const float *__restrict__ ufx,
                            const float *__restrict__ ufy, const float *__restrict__ ufz,
                            const float *__restrict__ sin_, const float *__restrict__ sout)
{
    Idx3s t = decode_s(g.nx + 1, g.nz + 1, g.ny + 1);
    if (!t.ok) return;
    const int i = t.i, k = t.k, j = t.j, nz = g.nz;
    const int is = its - 1, ie = ite + 1, js = jts - 1, je = jte + 1;
    const size_t sy = (size_t)g.P * g.nz, sz = (size_t)g.P;
    if (k < nz) {
        if (j >= js && j <= je && i >= is && i <= ie + 1) {
            size_t c = ix(g, i, k, j);
            float F = fx[c];
            if (i >= its && i <= ite + 1) {
                if (F > 0.0f) F = fmin_(sin_[c], sout[c - 1]) * F;
                else if (F < 0.0f) F = fmin_(sout[c], sin_[c - 1]) * F;
            }
            fx[c] = F + ufx[c];
        }
        if (i >= is && i <= ie && j >= js && j <= je + 1) {
            size_t c = ix(g, i, k, j);
            float F = fy[c];
            if (j >= jts && j <= jte + 1) {
                if (F > 0.0f) F = fmin_(sin_[c], sout[c - sy]) * F;
                else if (F < 0.0f) F = fmin_(sout[c], sin_[c - sy]) * F;
            }
            fy[c] = F + ufy[c];
        }
    }
    if (i >= is && i <= ie && j >= js && j <= je) {
        size_t zf = izf(g, i, k, j);
        float F = fz[zf];
        if (k >= 1 && k <= nz - 1) {
            size_t c = ix(g, i, k, j);
            if (F > 0.0f) F = fmin_(sin_[c], sout[c - sz]) * F;
            else if (F < 0.0f) F = fmin_(sout[c], sin_[c - sz]) * F;
        }
        fz[zf] = F + ufz[zf];
    }
}

}  // namespace icar
