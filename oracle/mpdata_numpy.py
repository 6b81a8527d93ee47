"""Second, independent restatement of ICAR's MPDATA advection: numpy, slice
for slice.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module; the
tests use it to cross-check the C oracle (icar_adv_oracle.c), so that a
misreading of the Fortran shared by the C oracle and the CUDA kernels (both
written from one reading) would show up as a disagreement here.  It shares
no code with the C oracle: every routine below transliterates the Fortran
array statements of src/physics/adv_mpdata.f90 and
src/physics/adv_mpdata_FCT_core.f90 statement by statement, with the
Fortran index ranges written out through the `F` indexer (inclusive bounds,
the declared lower bounds of each array), and numpy float32 arithmetic,
which rounds every operation to single precision like the `real` Fortran
code.  The per-line FCT sweep keeps its sequential loop over the line and
runs all lines of a direction at once as vectors (the lines are
independent: each carries its own qmax_i2/fin_i2).

Arrays live in numpy as (j, k, i) = (y, z, x), the memory order of the
Fortran (i, k, j) arrays.  The domain is one image: ims = kms = jms = 1,
ime = nx, kme = nz, jme = ny.
"""
from __future__ import annotations

import numpy as np

f4 = np.float32


class F:
    """View of a numpy (j, k, i) array addressed like Fortran a(i, k, j).

    `lb` are the declared lower bounds (i, k, j).  A slice `lo:hi` means the
    Fortran section lo:hi with hi INCLUSIVE; `:` is the whole extent."""

    def __init__(self, arr: np.ndarray, lb=(1, 1, 1)):
        self.a = arr
        self.lb = lb

    def _conv(self, key):
        out = []
        for d, kk in enumerate(key):
            lb = self.lb[d]
            if isinstance(kk, slice):
                lo = 0 if kk.start is None else kk.start - lb
                hi = None if kk.stop is None else kk.stop - lb + 1
                out.append(slice(lo, hi))
            else:
                out.append(kk - lb)
        return tuple(reversed(out))

    def __getitem__(self, key):
        return self.a[self._conv(key)]

    def __setitem__(self, key, val):
        self.a[self._conv(key)] = val


class V1:
    """1-D Fortran vector with a declared lower bound; inclusive slices."""

    def __init__(self, n_or_arr, lb: int):
        self.a = np.zeros(n_or_arr, f4) if isinstance(n_or_arr, int) else n_or_arr
        self.lb = lb

    def _s(self, kk):
        if isinstance(kk, slice):
            lo = 0 if kk.start is None else kk.start - self.lb
            hi = None if kk.stop is None else kk.stop - self.lb + 1
            return slice(lo, hi)
        return kk - self.lb

    def __getitem__(self, kk):
        return self.a[self._s(kk)]

    def __setitem__(self, kk, val):
        self.a[self._s(kk)] = val


class Bounds:
    def __init__(self, nx: int, ny: int, nz: int):
        self.ims, self.ime = 1, nx
        self.kms, self.kme = 1, nz
        self.jms, self.jme = 1, ny


def flux1(l, r, U):
    """adv_mpdata.f90:23-41: f = ((U+|U|)*l + (U-|U|)*r)/2."""
    return ((U + np.abs(U)) * l + (U - np.abs(U)) * r) / f4(2)


def upwind_advection(b: Bounds, qin: F, u: F, v: F, w: F, rho: F, q: F, dz: F, jaco: F):
    """adv_mpdata.f90:43-103.  u is declared (ims+1:ime, ...), v
    (ims:ime, kms:kme, jms+1:jme); q receives the result."""
    ims, ime, kms, kme, jms, jme = b.ims, b.ime, b.kms, b.kme, b.jms, b.jme
    for i in range(jms, jme + 1):                                            # :61-63
        q[:, :, i] = qin[:, :, i]
    for i in range(jms + 1, jme - 1 + 1):                                    # :68
        f1 = F(np.zeros((kme - kms + 1, ime - ims), f4)[None], (ims, kms, 0))   # f1(ims:ime-1, kms:kme)
        f1[ims:ime - 1, :, 0] = ((u[ims + 1:ime, :, i] + np.abs(u[ims + 1:ime, :, i])) * qin[ims:ime - 1, :, i] +
                                 (u[ims + 1:ime, :, i] - np.abs(u[ims + 1:ime, :, i])) * qin[ims + 1:ime, :, i]) / f4(2)
        f3 = ((v[ims + 1:ime - 1, :, i + 1] + np.abs(v[ims + 1:ime - 1, :, i + 1])) * qin[ims + 1:ime - 1, :, i] +
              (v[ims + 1:ime - 1, :, i + 1] - np.abs(v[ims + 1:ime - 1, :, i + 1])) * qin[ims + 1:ime - 1, :, i + 1]) / f4(2)
        f4_ = ((v[ims + 1:ime - 1, :, i] + np.abs(v[ims + 1:ime - 1, :, i])) * qin[ims + 1:ime - 1, :, i - 1] +
               (v[ims + 1:ime - 1, :, i] - np.abs(v[ims + 1:ime - 1, :, i])) * qin[ims + 1:ime - 1, :, i]) / f4(2)
        # f5(ims:ime-2, kms:kme-1): the x extent of the section is ims+1:ime-1
        f5 = F(np.zeros((kme - kms, ime - ims - 1), f4)[None], (ims, kms, 0))
        f5[:, :, 0] = ((w[ims + 1:ime - 1, kms:kme - 1, i] + np.abs(w[ims + 1:ime - 1, kms:kme - 1, i])) *
                       qin[ims + 1:ime - 1, kms:kme - 1, i] +
                       (w[ims + 1:ime - 1, kms:kme - 1, i] - np.abs(w[ims + 1:ime - 1, kms:kme - 1, i])) *
                       qin[ims + 1:ime - 1, kms + 1:kme, i]) / f4(2)
        # :86-87 horizontal
        q[ims + 1:ime - 1, :, i] = q[ims + 1:ime - 1, :, i] - ((f1[ims + 1:ime - 1, :, 0] - f1[ims:ime - 2, :, 0]) +
                                                              (f3 - f4_)) / (jaco[ims + 1:ime - 1, :, i] *
                                                                             rho[ims + 1:ime - 1, :, i])
        # :90-91 middle layers
        q[ims + 1:ime - 1, kms + 1:kme - 1, i] = q[ims + 1:ime - 1, kms + 1:kme - 1, i] - \
            (f5[:, kms + 1:kme - 1, 0] - f5[:, kms:kme - 2, 0]) / \
            (dz[ims + 1:ime - 1, kms + 1:kme - 1, i] * jaco[ims + 1:ime - 1, kms + 1:kme - 1, i] *
             rho[ims + 1:ime - 1, kms + 1:kme - 1, i])
        # :93-94 bottom
        q[ims + 1:ime - 1, kms, i] = q[ims + 1:ime - 1, kms, i] - f5[:, kms, 0] / \
            (dz[ims + 1:ime - 1, kms, i] * jaco[ims + 1:ime - 1, kms, i] * rho[ims + 1:ime - 1, kms, i])
        # :96-97 top
        q[ims + 1:ime - 1, kme, i] = q[ims + 1:ime - 1, kme, i] - \
            (qin[ims + 1:ime - 1, kme, i] * w[ims + 1:ime - 1, kme, i] - f5[:, kme - 1, 0]) / \
            (dz[ims + 1:ime - 1, kme, i] * jaco[ims + 1:ime - 1, kme, i] * rho[ims + 1:ime - 1, kme, i])


def mpdata_fluxes(b: Bounds, q: F, u: F, v: F, w: F, u2: F, v2: F, w2: F, G: F):
    """adv_mpdata.f90:105-252: antidiffusive pseudo-velocities u2
    (ims+1:ime, ...), v2 (..., jms+1:jme), w2 from q with the cross terms."""
    ims, ime, kms, kme, jms, jme = b.ims, b.ime, b.kms, b.kme, b.jms, b.jme
    e10 = f4(1e-10)
    u2.a[...] = 0
    v2.a[...] = 0
    w2.a[...] = 0
    for i in range(jms, jme + 1):
        for j in range(kms, kme + 1):
            # ---------------- U component (:131-166)
            if i > 0:
                rx = V1(q[ims + 1:ime, j, i].copy(), ims + 1)
                lx = V1(q[ims:ime - 1, j, i].copy(), ims + 1)
                denomx = rx.a + lx.a + e10
                u2[:, j, i] = np.abs(u[:, j, i]) * (f4(1) - np.abs(u[:, j, i]) /
                                                    (f4(0.5) * (G[ims + 1:ime, j, i] + G[ims:ime - 1, j, i])))
                u2[:, j, i] = u2[:, j, i] * (rx.a - lx.a) / denomx
                edge_v = V1(ime - ims + 1, ims)
                edge_q = V1(ime - ims + 1, ims)
                if (i > jms) and (i < jme):                                  # UxV
                    edge_q[ims + 1:ime] = (q[ims + 1:ime, j, i + 1] - q[ims + 1:ime, j, i - 1] +
                                           q[ims:ime - 1, j, i + 1] - q[ims:ime - 1, j, i - 1]) / \
                                          (q[ims + 1:ime, j, i + 1] + q[ims + 1:ime, j, i - 1] +
                                           q[ims:ime - 1, j, i + 1] + q[ims:ime - 1, j, i - 1] + e10)
                    edge_v[ims + 1:ime] = (f4(1) / f4(4.0)) * (v[ims + 1:ime, j, i] + v[ims + 1:ime, j, i + 1] +
                                                               v[ims:ime - 1, j, i] + v[ims:ime - 1, j, i + 1])
                    u2[:, j, i] = u2[:, j, i] - f4(0.5) * u[:, j, i] * edge_v[ims + 1:ime] * edge_q[ims + 1:ime] / \
                        (G[ims + 1:ime, j, i] + G[ims:ime - 1, j, i])
                edge_v = V1(ime - ims + 1, ims)
                edge_q = V1(ime - ims + 1, ims)
                if (j > kms) and (j < kme):                                  # UxW
                    edge_q[ims + 1:ime] = (q[ims + 1:ime, j + 1, i] - q[ims + 1:ime, j - 1, i] +
                                           q[ims:ime - 1, j + 1, i] - q[ims:ime - 1, j - 1, i]) / \
                                          (q[ims + 1:ime, j + 1, i] + q[ims + 1:ime, j - 1, i] +
                                           q[ims:ime - 1, j + 1, i] + q[ims:ime - 1, j - 1, i] + e10)
                    edge_v[ims + 1:ime] = (f4(1) / f4(4.0)) * (w[ims + 1:ime, j, i] + w[ims + 1:ime, j - 1, i] +
                                                               w[ims:ime - 1, j, i] + w[ims:ime - 1, j - 1, i])
                    u2[:, j, i] = u2[:, j, i] - f4(0.5) * u[:, j, i] * edge_v[ims + 1:ime] * edge_q[ims + 1:ime] / \
                        (G[ims + 1:ime, j, i] + G[ims:ime - 1, j, i])
            # ---------------- V component (:170-206)
            if i > jms:
                r = q[:, j, i].copy()
                l = q[:, j, i - 1].copy()
                denom = r + l + e10
                v2[:, j, i] = np.abs(v[:, j, i]) * (f4(1) - np.abs(v[:, j, i]) /
                                                    (f4(0.5) * (G[:, j, i] + G[:, j, i - 1])))
                v2[:, j, i] = v2[:, j, i] * (r - l) / denom
                edge_v = V1(ime - ims + 1, ims)
                edge_q = V1(ime - ims + 1, ims)
                edge_q[ims + 1:ime - 1] = (q[ims + 2:ime, j, i - 1] - q[ims:ime - 2, j, i] +
                                           q[ims + 2:ime, j, i] - q[ims:ime - 2, j, i - 1]) / \
                                          (q[ims + 2:ime, j, i] + q[ims + 2:ime, j, i - 1] +
                                           q[ims:ime - 2, j, i] + q[ims:ime - 2, j, i - 1] + e10)
                edge_v[ims + 1:ime - 1] = (f4(1) / f4(4.0)) * \
                    (u[ims + 2:ime, j, i] + u[ims + 2:ime, j, i - 1] + u[ims + 1:ime - 1, j, i] + u[ims + 1:ime - 1, j, i - 1])
                v2[:, j, i] = v2[:, j, i] - f4(0.5) * v[:, j, i] * edge_v.a * edge_q.a / (G[:, j, i] + G[:, j, i - 1])
                edge_v = V1(ime - ims + 1, ims)
                edge_q = V1(ime - ims + 1, ims)
                if (j > kms) and (j < kme):                                  # VxW
                    edge_q.a = (q[:, j + 1, i - 1] - q[:, j - 1, i] + q[:, j + 1, i] - q[:, j - 1, i - 1]) / \
                               (q[:, j + 1, i - 1] + q[:, j - 1, i] + q[:, j + 1, i] + q[:, j - 1, i - 1] + e10)
                    edge_v.a = (f4(1) / f4(4.0)) * (w[:, j, i] + w[:, j - 1, i] + w[:, j, i - 1] + w[:, j - 1, i - 1])
                    v2[:, j, i] = v2[:, j, i] - f4(0.5) * v[:, j, i] * edge_v.a * edge_q.a / (G[:, j, i] + G[:, j, i - 1])
            # ---------------- W component (:211-247)
            if j == kme:
                w2[:, j, i] = 0
            else:
                r = q[:, j + 1, i].copy()
                l = q[:, j, i].copy()
                denom = r + l + e10
                w2[:, j, i] = np.abs(w[:, j, i]) * (f4(1) - np.abs(w[:, j, i]) /
                                                    (f4(0.5) * (G[:, j + 1, i] + G[:, j, i])))
                w2[:, j, i] = w2[:, j, i] * (r - l) / denom
                edge_v = V1(ime - ims + 1, ims)
                edge_q = V1(ime - ims + 1, ims)
                edge_q[ims + 1:ime - 1] = (q[ims + 2:ime, j + 1, i] - q[ims:ime - 2, j, i] +
                                           q[ims + 2:ime, j, i] - q[ims:ime - 2, j + 1, i]) / \
                                          (q[ims + 2:ime, j, i] + q[ims + 2:ime, j + 1, i] +
                                           q[ims:ime - 2, j, i] + q[ims:ime - 2, j + 1, i] + e10)
                edge_v[ims + 1:ime - 1] = (f4(1) / f4(4.0)) * \
                    (u[ims + 2:ime, j, i] + u[ims + 2:ime, j + 1, i] + u[ims + 1:ime - 1, j, i] + u[ims + 1:ime - 1, j + 1, i])
                w2[:, j, i] = w2[:, j, i] - f4(0.5) * w[:, j, i] * edge_v.a * edge_q.a / (G[:, j + 1, i] + G[:, j, i])
                edge_v = V1(ime - ims + 1, ims)
                edge_q = V1(ime - ims + 1, ims)
                if (i > jms) and (i < jme):                                  # WxV
                    edge_q.a = (q[:, j + 1, i + 1] - q[:, j, i - 1] + q[:, j, i + 1] - q[:, j + 1, i - 1]) / \
                               (q[:, j, i + 1] + q[:, j + 1, i - 1] + q[:, j + 1, i + 1] + q[:, j, i - 1] + e10)
                    edge_v.a = (f4(1) / f4(4.0)) * (v[:, j, i] + v[:, j + 1, i] + v[:, j, i + 1] + v[:, j + 1, i + 1])
                    w2[:, j, i] = w2[:, j, i] - f4(0.5) * w[:, j, i] * edge_v.a * edge_q.a / (G[:, j + 1, i] + G[:, j, i])


def fct_core(q1: np.ndarray, l: np.ndarray, U2: np.ndarray, f: np.ndarray, n_s: int, n: int, flux_is_w: bool):
    """adv_mpdata_FCT_core.f90:47-116 on a set of independent lines at once.

    The last axis is the line (Fortran index n_s..n); q1 and l have n-n_s+1
    points, U2 and f n-n_s (faces n_s..n-1, face i between cells i and
    i+1).  U2 is limited in place.  The scalars of the Fortran loop
    (qmax_i, fin_i2, beta_*, ...) are vectors over the lines."""
    def at(a, i):
        return a[..., i - n_s]

    zero = f4(0.0)
    e15 = f4(1e-15)
    qmax_i2 = qmin_i2 = fin_i2 = fout_i2 = None
    for i in range(n_s, n - 1 + 1):
        if i == n_s:
            qmax_i = np.maximum.reduce([at(q1, i), at(q1, i + 1), at(l, i), at(l, i + 1)])
            qmin_i = np.minimum.reduce([at(q1, i), at(q1, i + 1), at(l, i), at(l, i + 1)])
            qmax_i2 = np.maximum.reduce([at(q1, i), at(q1, i + 1), at(q1, i + 2), at(l, i), at(l, i + 1), at(l, i + 2)])
            qmin_i2 = np.minimum.reduce([at(q1, i), at(q1, i + 1), at(q1, i + 2), at(l, i), at(l, i + 1), at(l, i + 2)])
        elif i != (n - 1):
            qmax_i = qmax_i2
            qmin_i = qmin_i2
            qmax_i2 = np.maximum.reduce([at(q1, i), at(q1, i + 1), at(q1, i + 2), at(l, i), at(l, i + 1), at(l, i + 2)])
            qmin_i2 = np.minimum.reduce([at(q1, i), at(q1, i + 1), at(q1, i + 2), at(l, i), at(l, i + 1), at(l, i + 2)])
        else:
            qmax_i = qmax_i2
            qmin_i = qmin_i2
            qmax_i2 = np.maximum.reduce([at(q1, i), at(q1, i + 1), at(l, i)])
            qmin_i2 = np.minimum.reduce([at(q1, i), at(q1, i + 1), at(l, i)])
        fi = at(f, i)
        if i != n_s:
            fin_i = fin_i2
            fout_i = fout_i2
        else:
            if flux_is_w:
                fin_i = zero - np.minimum(zero, fi)
                fout_i = np.maximum(zero, fi)
            else:
                fin_i = np.zeros_like(fi)
                fout_i = np.zeros_like(fi)
        if i != (n - 1):
            fi1 = at(f, i + 1)
            fin_i2 = np.maximum(zero, fi) - np.minimum(zero, fi1)
            fout_i2 = np.maximum(zero, fi1) - np.minimum(zero, fi)
        else:
            if flux_is_w:
                fin_i2 = np.maximum(zero, fi) - np.minimum(zero, fi)
                fout_i2 = np.maximum(zero, fi) - np.minimum(zero, fi)
            else:
                fin_i2 = np.zeros_like(fi)
                fout_i2 = np.zeros_like(fi)
        u = at(U2, i)
        with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
            beta_out_i = (at(q1, i) - qmin_i) / (fout_i + e15)
            beta_in_i2 = (qmax_i2 - at(q1, i + 1)) / (fin_i2 + e15)
            beta_in_i = (qmax_i - at(q1, i)) / (fin_i + e15)
            beta_out_i2 = (at(q1, i + 1) - qmin_i2) / (fout_i2 + e15)
        pos = np.minimum.reduce([np.full_like(u, 1.0), beta_in_i2, beta_out_i]) * u
        neg = np.minimum.reduce([np.full_like(u, 1.0), beta_in_i, beta_out_i2]) * u
        U2[..., i - n_s] = np.where(u > 0, pos, np.where(u < 0, neg, u))


def flux_limiter(b: Bounds, q: F, q2: F, u: F, v: F, w: F):
    """adv_mpdata.f90:254-350.  The dummies re-declare the actual arrays'
    bounds: u is (ims:ime-1, ...) over the actual u2 (ims+1:ime, ...), so
    u(i) is the face between cells i and i+1; v is (..., jms:jme-1) over v2
    (..., jms+1:jme)."""
    ims, ime, kms, kme, jms, jme = b.ims, b.ime, b.kms, b.kme, b.jms, b.jme
    uu = F(u.a, (ims, kms, jms))            # re-declared lower bound ims
    vv = F(v.a, (ims, kms, jms))            # re-declared lower bound jms
    # x lines: rows j = jms+1..jme-1, every k (:283-300)
    rows = slice(jms + 1 - 1, jme - 1)
    q1 = q2.a[rows]                          # (rows, nz, nx): lines along the last axis
    l = q.a[rows]
    U2 = uu.a[rows].copy()
    f = flux1(q1[..., :-1], q1[..., 1:], U2)
    fct_core(q1, l, U2, f, ims, ime, False)
    uu.a[rows] = U2
    # z lines: rows j = jms+1..jme-1, columns ims+1..ime-1 (:302-319)
    cols = slice(ims + 1 - 1, ime - 1)
    q1 = np.moveaxis(q2.a[rows][:, :, cols], 1, 2)          # (rows, cols, nz)
    l = np.moveaxis(q.a[rows][:, :, cols], 1, 2)
    U2 = np.moveaxis(w.a[rows][:, kms - 1:kme - 1, cols], 1, 2).copy()
    f = flux1(q1[..., :-1], q1[..., 1:], U2)
    fct_core(q1, l, U2, f, kms, kme, True)
    wr = w.a[rows]
    wr[:, kms - 1:kme - 1, cols] = np.moveaxis(U2, 2, 1)
    wr[:, kme - 1, cols] = 0
    w.a[rows] = wr
    # y lines: every column and level (:336-346)
    q1 = np.moveaxis(q2.a, 0, 2)                            # (nz, nx, ny)
    l = np.moveaxis(q.a, 0, 2)
    U2 = np.moveaxis(vv.a, 0, 2).copy()
    f = flux1(q1[..., :-1], q1[..., 1:], U2)
    fct_core(q1, l, U2, f, jms, jme, False)
    vv.a[...] = np.moveaxis(U2, 2, 0)


def mpdata_advect3d(b: Bounds, q: F, rho: F, jaco: F, dz: F, U_m: F, V_m: F, W_m: F, mpdata_order: int,
                    mpdata_fct: bool):
    """adv_mpdata.f90:352-413 (rho is domain%density, the real density)."""
    nx, nz, ny = b.ime, b.kme, b.jme
    q2 = F(np.zeros((ny, nz, nx), f4))
    u2 = F(np.zeros((ny, nz, nx - 1), f4), (2, 1, 1))
    v2 = F(np.zeros((ny - 1, nz, nx), f4), (1, 1, 2))
    w2 = F(np.zeros((ny, nz, nx), f4))
    for iord in range(1, mpdata_order + 1):
        if iord == 1:
            upwind_advection(b, q, U_m, V_m, W_m, rho, q2, dz, jaco)
        else:
            wdz = F(W_m.a / dz.a)
            G = F(jaco.a * rho.a)
            mpdata_fluxes(b, q2, U_m, V_m, wdz, u2, v2, w2, G)
            u2.a[...] = u2.a * f4(0.5)
            v2.a[...] = v2.a * f4(0.5)
            w2.a[...] = w2.a * f4(0.5) * dz.a
            if mpdata_fct:
                flux_limiter(b, q, q2, u2, v2, w2)
            upwind_advection(b, q2, u2, v2, w2, rho, q, dz, jaco)
        if iord != mpdata_order:
            if iord > 1:
                q2.a[...] = q.a
        else:
            if iord == 1:
                q.a[...] = q2.a


def mpdata_compute_wind(b: Bounds, u: F, v: F, w: F, density: F, jacobian_u: F, jacobian_v: F, jacobian_w: F,
                        dx: float, dt: float, advect_density: bool):
    """adv_mpdata.f90:477-504; returns U_m (ims+1:ime), V_m (jms+1:jme), W_m."""
    ims, ime, kms, kme, jms, jme = b.ims, b.ime, b.kms, b.kme, b.jms, b.jme
    dx, dt = f4(dx), f4(dt)
    rho = F(np.ones_like(density.a))
    if advect_density:
        rho.a[...] = density.a
    U_m = F(np.zeros((jme, kme, ime - ims), f4), (ims + 1, kms, jms))
    V_m = F(np.zeros((jme - jms, kme, ime), f4), (ims, kms, jms + 1))
    W_m = F(np.zeros((jme, kme, ime), f4))
    U_m.a[...] = u[ims + 1:ime, :, :] * dt * (rho[ims + 1:ime, :, :] + rho[ims:ime - 1, :, :]) * f4(0.5) * \
        jacobian_u[ims + 1:ime, :, :] / dx
    V_m.a[...] = v[:, :, jms + 1:jme] * dt * (rho[:, :, jms + 1:jme] + rho[:, :, jms:jme - 1]) * f4(0.5) * \
        jacobian_v[:, :, jms + 1:jme] / dx
    W_m[:, kms:kme - 1, :] = w[:, kms:kme - 1, :] * dt * jacobian_w[:, kms:kme - 1, :] * \
        (rho[:, kms + 1:kme, :] + rho[:, kms:kme - 1, :]) * f4(0.5)
    W_m[:, kme, :] = w[:, kme, :] * dt * jacobian_w[:, kme, :] * rho[:, kme, :]
    return U_m, V_m, W_m


def advect(case, dt: float, mpdata_order: int = 2, mpdata_fct: bool = True, advect_density: bool = False) -> dict:
    """advect(domain, options, dt) for MPDATA without RK3
    (advection_driver.f90:59-126): winds once, then every species in
    adv_vars order.  Returns new float32 arrays (the case is not modified)."""
    nx, ny, nz = case.nx, case.ny, case.nz
    b = Bounds(nx, ny, nz)
    a = lambda k: np.ascontiguousarray(getattr(case, k), dtype=f4)
    u = F(a("u"))                      # u%data_3d(ims:ime+1, ...)
    v = F(a("v"))                      # v%data_3d(..., jms:jme+1)
    U_m, V_m, W_m = mpdata_compute_wind(b, u, v, F(a("w")), F(a("density")), F(a("jacobian_u")),
                                        F(a("jacobian_v")), F(a("jacobian_w")), case.dx, dt, advect_density)
    out = {}
    for name, q in case.species.items():
        qq = F(np.ascontiguousarray(q, dtype=f4).copy())
        mpdata_advect3d(b, qq, F(a("density")), F(a("jacobian")), F(a("advection_dz")), U_m, V_m, W_m,
                        mpdata_order, mpdata_fct)
        out[name] = qq.a
    return out
