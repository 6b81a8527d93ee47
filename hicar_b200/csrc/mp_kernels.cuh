// Simple microphysics (SB04) on the device: mp_simple_driver,
// src/physics/mp_simple.f90:595-646, the scheme mp_driver.f90:548-568 runs
// after advection when physics%microphysics = kMP_SB04.
//
// k_mp_simple: one thread per column of the tile (its..ite x jts..jte).
// Phase 1 walks up the column doing the per-level conversions
// (mp_conversions: saturation adjustment by the reference's iteration,
// autoconversion, melting, evaporation and sublimation with latent-heat
// feedback), its inputs arriving in shared-memory planes by cp.async three
// levels ahead; it leaves the air temperature T = th*pii in the th array
// and forms on the way the column maxima the sedimentation passes start
// from (in the reference's order, level 0 first).
// Phases 2 and 3 sediment rain and then snow in CFL substeps (sediment, as a
// single upward sweep: each level's downward flux is formed from the level
// above before that level is touched, exactly the reference's values and
// order) with the evaporation/sublimation of what fell into unsaturated
// levels.  Phase 4 turns T back into th.  With one substep each (the usual
// case) phases 2-4 run as a second staged march, level by level (see the
// kernel).  The column's rain and snow are added to the real64
// accumulations (one writer per column).
//
// Arithmetic follows the reference expression by expression (no FMA
// contraction).  The one transcendental, exp in sat_mr, is evaluated as the
// float rounding of a double-precision exp: the correctly rounded
// single-precision exp except within about 2^-29 ulp of a halfway point.
// The CPU restatement evaluates it the same way; the reference's libm expf
// may differ from it in the last bit in near-halfway cases.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"
#include "mpdata_fused.cuh"

namespace icar {
namespace mps {
constexpr float LH_VAPOR = 2.26E6f, DLHVDT = 2400.0f, LH_LIQUID = 3.34E5f, HEAT_CAPACITY = 1006.0f;
constexpr float SMALL = 1E-30f, FREEZING = 273.15f;
constexpr float SNOW_FALL = 1.5f, RAIN_FALL = 10.0f, SNOW_INIT = 0.0001f, RAIN_INIT = 0.0001f;
}  // namespace mps

// sat_mr, mp_simple.f90:146-182
__device__ __forceinline__ float mp_sat_mr(float temperature, float pressure)
{
    float a, b;
    if (temperature < mps::FREEZING) {
        a = 21.8745584f;
        b = 7.66f;
    } else {
        a = 17.2693882f;
        b = 35.86f;
    }
    float e_s = 610.78f * __double2float_rn(exp((double)(a * (temperature - 273.16f) / (temperature - b))));
    if ((pressure - e_s) <= 0.0f) e_s = pressure * 0.99999f;
    return 0.6219907f * e_s / (pressure - e_s);
}

// cloud_conversion, mp_simple.f90:198-280 (its diagnostic prints omitted)
__device__ __forceinline__ void mp_cloud_conversion(float pressure, float &temperature, float &qv, float &qc,
                                                    float &qvsat)
{
    const float maxerr = 1e-4f;
    int iteration = 0;
    float lastqv = qv + maxerr * 2.0f;
    const float vapor2temp = (mps::LH_VAPOR + (373.15f - temperature) * mps::DLHVDT) / mps::HEAT_CAPACITY;
    const float pre_qc = qc, pre_t = temperature;
    while ((fabsf(lastqv - qv) > maxerr) && (iteration < 15)) {
        iteration = iteration + 1;
        lastqv = qv;
        qvsat = mp_sat_mr(temperature, pressure);
        if (qv > qvsat) {
            const float excess = (qv - qvsat) * 0.5f;
            temperature = temperature + (excess * vapor2temp);
            qv = qv - excess;
            qc = qc + excess;
        } else if (qc > 0.0f) {
            const float excess = (qvsat - qv) * 0.5f;
            if (excess < qc) {
                temperature = temperature - (excess * vapor2temp);
                qv = qv + excess;
                qc = qc - excess;
            } else {
                qv = qv + qc;
                temperature = temperature - (qc * vapor2temp);
                qc = 0.0f;
            }
        }
    }
    if (iteration == 15) {
        qv = mp_sat_mr(pre_t, pressure);
        temperature = pre_t;
        qc = pre_qc;
    }
    qc = fmax_(qc, 0.0f);
}

// cloud2hydrometeor, mp_simple.f90:295-315
__device__ __forceinline__ void mp_cloud2hydrometeor(float &qc, float &q, float conversion, float qcmin)
{
    const float delta = qc > qcmin ? qc - (qc * conversion) : 0.0f;
    if (delta < qc) {
        qc = qc - delta;
        q = q + delta;
    } else {
        q = q + qc;
        qc = 0.0f;
    }
    qc = fmax_(qc, 0.0f);
}

// phase_change, mp_simple.f90:333-362; stop is set where the reference
// stops the program (q1 left in [-1e-30, 0))
__device__ __forceinline__ void mp_phase_change(float &temperature, float &q1, float qmax, float &q2, float Lheat,
                                                float change_rate, int &stop)
{
    const float mass2temp = Lheat / mps::HEAT_CAPACITY;
    float delta = (qmax - q2) * change_rate;
    if (delta > q1) delta = q1;
    if (delta > ((qmax - q2) * 0.99f)) delta = (qmax - q2) * 0.99f;
    q1 = q1 - delta;
    if (q1 < 0.0f) {
        if ((q1 + mps::SMALL) < 0.0f)
            q1 = 0.0f;
        else
            stop = 1;
    }
    q2 = q2 + delta;
    temperature = temperature + delta * mass2temp;
}

// mp_conversions, mp_simple.f90:381-420
__device__ __forceinline__ void mp_conversions(float pressure, float &temperature, float &qv, float &qc, float &qr,
                                               float &qs, float cloud2rain, float cloud2snow, int &stop)
{
    const float L_melt = -1.0f * mps::LH_LIQUID;
    const float L_evap = -1.0f * (mps::LH_VAPOR + (373.15f - temperature) * mps::DLHVDT);
    const float L_subl = L_melt + L_evap;
    float qvsat = 0.0f;
    mp_cloud_conversion(pressure, temperature, qv, qc, qvsat);
    if ((qc + qr + qs) > mps::SMALL) {
        if (qc > mps::SMALL) {
            if (temperature > mps::FREEZING) {
                mp_cloud2hydrometeor(qc, qr, cloud2rain, mps::RAIN_INIT);
                if (qs > mps::SMALL) mp_phase_change(temperature, qs, 100.0f, qr, L_melt, cloud2rain, stop);
            } else {
                mp_cloud2hydrometeor(qc, qs, cloud2snow, mps::SNOW_INIT);
            }
        }
        if (qv < qvsat) {
            if (qr > mps::SMALL) mp_phase_change(temperature, qr, qvsat, qv, L_evap, cloud2rain / 2.0f, stop);
            if (qs > mps::SMALL) mp_phase_change(temperature, qs, qvsat, qv, L_subl, cloud2snow / 2.0f, stop);
        }
    }
}

namespace mpsf {
// CTA tile of 32 x 4 columns; the planes of one level span x from
// floor4(i0) to +35 (a multiple of 4, so 16-byte chunks).
constexpr int BX = 32, BY = 4, NT = BX * BY;
constexpr int PW = 36, PH = BY, PLANE = PW * PH;   // x from floor4(i0) to +35
constexpr int NF = 8;                               // pressure, th, pii, qv, qc, qr, qs, dz
constexpr int DEPTH = 3, NSLOT = DEPTH + 1;
constexpr int CPR = PW / 4, NCH = (NF * CPR * PH + NT - 1) / NT;
constexpr size_t SMEM = (size_t)NSLOT * NF * PLANE * sizeof(float);
}  // namespace mpsf

// One column per thread; phase 1 reads its levels from shared-memory planes
// filled by cp.async ahead of use.  T lives in th between the phases.
__global__ void __launch_bounds__(mpsf::NT)
    k_mp_simple(Geo g, int hs, float dt, float cloud2rain, float cloud2snow,
                const float *__restrict__ pressure, float *__restrict__ th, const float *__restrict__ pii,
                const float *__restrict__ rho, float *__restrict__ qv, float *__restrict__ qc,
                float *__restrict__ qr, float *__restrict__ qs, const float *__restrict__ dz,
                double *__restrict__ acc_rain, double *__restrict__ acc_snow, int *__restrict__ stop_flag)
{
    using namespace mpsf;
    extern __shared__ float4 sm4[];
    float *sm = reinterpret_cast<float *>(sm4);
    const int tx = threadIdx.x % BX, ty = threadIdx.x / BX;
    const int i0 = hs + blockIdx.x * BX, j0 = hs + blockIdx.y * BY;
    const int i = i0 + tx, j = j0 + ty;
    const int ox = i0 - (i0 & 3), oy = j0;
    const bool col = i < g.nx - hs && j < g.ny - hs;
    const int nz = g.nz;
    const size_t st = (size_t)g.P, c0 = col ? ix(g, i, 0, j) : 0;
    int stop = 0;
    const float *src[NCH];
    size_t off[NCH];
    int dst[NCH], fld[NCH];
    bool ok[NCH];
#pragma unroll
    for (int c = 0; c < NCH; c++) {
        const int e = threadIdx.x + c * NT;
        dst[c] = -1;
        fld[c] = 0;
        ok[c] = false;
        off[c] = 0;
        src[c] = pressure;
        if (e < NF * CPR * PH) {
            const int f = e / (CPR * PH), r = e % (CPR * PH);
            const int ly = r / CPR, cx = r % CPR;
            const int gi = ox + 4 * cx, gj = oy + ly;
            dst[c] = f * PLANE + ly * PW + 4 * cx;
            fld[c] = f;
            // phase 1 planes: pressure, th, pii, qv, qc, qr, qs, dz
            src[c] = f == 0 ? pressure : f == 1 ? th : f == 2 ? pii : f == 3 ? qv : f == 4 ? qc : f == 5 ? qr : f == 6 ? qs : dz;
            ok[c] = gi < g.P && gj < g.ny;
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
    const int pc = ty * PW + (i - ox);
    // column maxima the sedimentation passes start from, formed in the
    // reference's order (level 0 first) while the levels go by
    float mx_r = 0.0f, mx_s = 0.0f, m_r = 0.0f, m_s = 0.0f;
    // phase 1: conversions level by level
    for (int k = 0; k < nz; k++) {
        cp_async_wait<DEPTH - 1>();
        __syncthreads();
        issue(k + DEPTH);
        if (!col) continue;
        const float *L = sm + (size_t)(k % NSLOT) * NF * PLANE + pc;
        const size_t c = c0 + k * st;
        float T = L[PLANE] * L[2 * PLANE];
        float v = L[3 * PLANE], cw = L[4 * PLANE], r = L[5 * PLANE], s = L[6 * PLANE];
        mp_conversions(L[0], T, v, cw, r, s, cloud2rain, cloud2snow, stop);
        const float dzk = dt / L[7 * PLANE];
        if (k == 0) {
            mx_r = r;
            mx_s = s;
            m_r = dzk * mps::RAIN_FALL;
            m_s = dzk * mps::SNOW_FALL;
        } else {
            mx_r = fmax_(mx_r, r);
            mx_s = fmax_(mx_s, s);
            m_r = fmax_(m_r, dzk * mps::RAIN_FALL);
            m_s = fmax_(m_s, dzk * mps::SNOW_FALL);
        }
        th[c] = T;
        qv[c] = v;
        qc[c] = cw;
        qr[c] = r;
        qs[c] = s;
    }
    cp_async_wait<0>();
    __syncthreads();  // phase 1's results are in global memory for the planes below

    // Sedimentation parameters (the reference's expressions).  A column
    // whose rain and snow each take at most one substep runs phases 2-4 as
    // one more upward march over staged planes: at level k the rain and
    // snow sweeps finalise that level (each level's downward flux comes from
    // the level above), then rain evaporates and snow sublimates there and
    // th = T/pii is formed.  Every operation at level k reads and writes
    // level k only, apart from the sweeps' carried values, so the values
    // and their order are those of the separate passes.  Columns with more
    // substeps take the passes below.
    float fr_r = 0.0f, rate_r = 0.0f, fr_s = 0.0f, rate_s = 0.0f;
    int ns_r = 0, ns_s = 0;
    if (col && mx_r > mps::SMALL) {
        const float cfl = ceilf(m_r);
        fr_r = dt * mps::RAIN_FALL / cfl;
        ns_r = (int)lrintf(cfl);
        rate_r = cloud2rain / (float)(2 * ns_r);
    }
    if (col && mx_s > mps::SMALL) {
        const float cfl = ceilf(m_s);
        fr_s = dt * mps::SNOW_FALL / cfl;
        ns_s = (int)lrintf(cfl);
        rate_s = cloud2snow / (float)(2 * ns_s);
    }
    const bool fused = col && ns_r <= 1 && ns_s <= 1;
    // march 2 planes: th (T), qv, pressure, pii, qr, qs, rho, dz
#pragma unroll
    for (int c = 0; c < NCH; c++) {
        const int f = fld[c];
        src[c] = f == 0 ? th : f == 1 ? qv : f == 2 ? pressure : f == 3 ? pii : f == 4 ? qr : f == 5 ? qs : f == 6 ? rho : dz;
    }
#pragma unroll
    for (int k = 0; k < DEPTH; k++) issue(k);
    float qi_r = 0.0f, qi_s = 0.0f, sed_r = 0.0f, sed_s = 0.0f;
    for (int k = 0; k < nz; k++) {
        cp_async_wait<DEPTH - 2>();  // levels k and k+1 have landed
        __syncthreads();
        issue(k + DEPTH);            // into the slot of level k-1
        if (!fused) continue;
        const float *L = sm + (size_t)(k % NSLOT) * NF * PLANE + pc;
        const float *Lu = sm + (size_t)((k + 1) % NSLOT) * NF * PLANE + pc;
        const size_t c = c0 + k * st;
        if (k == 0) {
            // sediment out of the bottom level
            if (ns_r == 1) {
                qi_r = L[4 * PLANE];
                sed_r = fr_r * qi_r * L[6 * PLANE];
                qi_r = qi_r - (sed_r / L[7 * PLANE] / L[6 * PLANE]);
            }
            if (ns_s == 1) {
                qi_s = L[5 * PLANE];
                sed_s = fr_s * qi_s * L[6 * PLANE];
                qi_s = qi_s - (sed_s / L[7 * PLANE] / L[6 * PLANE]);
            }
        }
        float r = L[4 * PLANE], sn = L[5 * PLANE];
        if (ns_r == 1) {
            if (k < nz - 1) {
                float qu = Lu[4 * PLANE];
                const float ru = Lu[6 * PLANE];
                const float flux = fr_r * qu * ru;
                qi_r = qi_r + flux / (L[6 * PLANE] * L[7 * PLANE]);
                qu = qu - flux / (ru * Lu[7 * PLANE]);
                r = qi_r;
                qi_r = qu;
            } else {
                r = qi_r;
            }
        }
        if (ns_s == 1) {
            if (k < nz - 1) {
                float qu = Lu[5 * PLANE];
                const float ru = Lu[6 * PLANE];
                const float flux = fr_s * qu * ru;
                qi_s = qi_s + flux / (L[6 * PLANE] * L[7 * PLANE]);
                qu = qu - flux / (ru * Lu[7 * PLANE]);
                sn = qi_s;
                qi_s = qu;
            } else {
                sn = qi_s;
            }
        }
        float T = L[0], v = L[PLANE];
        const float p = L[2 * PLANE];
        if (ns_r == 1 && r > mps::SMALL) {
            const float L_evap = -1.0f * (mps::LH_VAPOR + (373.15f - T) * mps::DLHVDT);
            const float qvsat = mp_sat_mr(T, p);
            if (v < qvsat) mp_phase_change(T, r, qvsat, v, L_evap, rate_r, stop);
        }
        if (ns_s == 1 && sn > mps::SMALL) {
            const float L_evap = -1.0f * (mps::LH_VAPOR + (373.15f - T) * mps::DLHVDT);
            const float qvsat = mp_sat_mr(T, p);
            if (v < qvsat) mp_phase_change(T, sn, qvsat, v, -1.0f * mps::LH_LIQUID + L_evap, rate_s, stop);
        }
        th[c] = T / L[3 * PLANE];
        qv[c] = v;
        qr[c] = r;
        qs[c] = sn;
    }
    cp_async_wait<0>();
    if (!col) return;
    if (fused) {
        float rain = 0.0f, snow = 0.0f;
        if (ns_r == 1) rain = rain + sed_r;
        if (ns_s == 1) {
            snow = snow + sed_s;
            rain = rain + sed_s;
        }
        const size_t c2 = (size_t)i + (size_t)g.nx * j;
        acc_rain[c2] = acc_rain[c2] + (double)rain;
        acc_snow[c2] = acc_snow[c2] + (double)snow;
        if (stop) atomicOr(stop_flag, 1);
        return;
    }
    float rain = 0.0f, snow = 0.0f;
    // phases 2 and 3: sedimentation of rain, then of snow
    for (int pass = 0; pass < 2; pass++) {
        float *__restrict__ q = pass == 0 ? qr : qs;
        const float fall = pass == 0 ? mps::RAIN_FALL : mps::SNOW_FALL;
        const float mx = pass == 0 ? mx_r : mx_s;
        if (!(mx > mps::SMALL)) continue;
        const float m = pass == 0 ? m_r : m_s;
        const float cfl = ceilf(m);
        const float fall_rate = dt * fall / cfl;
        const int nsub = (int)lrintf(cfl);
        const float rate = (pass == 0 ? cloud2rain : cloud2snow) / (float)(2 * nsub);
        for (int sub = 0; sub < nsub; sub++) {
            // sediment: out of the bottom level, then one sweep of the
            // downward fluxes between levels i+1 -> i
            float qi = q[c0];
            const float sed = fall_rate * qi * rho[c0];
            qi = qi - (sed / dz[c0] / rho[c0]);
            for (int k = 0; k < nz - 1; k++) {
                const size_t c = c0 + k * st, cu = c + st;
                float qu = q[cu];
                const float ru = rho[cu];
                const float flux = fall_rate * qu * ru;
                qi = qi + flux / (rho[c] * dz[c]);
                qu = qu - flux / (ru * dz[cu]);
                q[c] = qi;
                qi = qu;
            }
            q[c0 + (size_t)(nz - 1) * st] = qi;
            if (pass == 0) {
                rain = rain + sed;
            } else {
                snow = snow + sed;
                rain = rain + sed;
            }
            // evaporate / sublimate what reached unsaturated levels; the
            // saturation mixing ratio is only formed where there is
            // something to evaporate (it has no other effect)
            for (int k = 0; k < nz; k++) {
                const size_t c = c0 + k * st;
                float h = q[c];
                if (!(h > mps::SMALL)) continue;
                float T = th[c];
                const float L_evap = -1.0f * (mps::LH_VAPOR + (373.15f - T) * mps::DLHVDT);
                const float qvsat = mp_sat_mr(T, pressure[c]);
                float v = qv[c];
                if (v < qvsat) {
                    mp_phase_change(T, h, qvsat, v, pass == 0 ? L_evap : -1.0f * mps::LH_LIQUID + L_evap, rate,
                                    stop);
                    th[c] = T;
                    qv[c] = v;
                    q[c] = h;
                }
            }
        }
    }
    // phase 4: back to potential temperature
    for (int k = 0; k < nz; k++) th[c0 + k * st] = th[c0 + k * st] / pii[c0 + k * st];
    const size_t c2 = (size_t)i + (size_t)g.nx * j;
    acc_rain[c2] = acc_rain[c2] + (double)rain;
    acc_snow[c2] = acc_snow[c2] + (double)snow;
    if (stop) atomicOr(stop_flag, 1);
}

}  // namespace icar
