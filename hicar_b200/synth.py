"""Seeded synthetic domains for the advection step.

The reference's benchmarks use real forcing data; here every input is
generated from a seed with the shapes and value distributions of the
workloads (terrain, terrain-following jacobians, winds with w from discrete
continuity, density and up to 12 advected fields).  Arrays use the Fortran
memory layout of domain_t as numpy C-order arrays:
    cell fields    (ny, nz, nx)      <->  Fortran (nx, nz, ny)
    u-grid fields  (ny, nz, nx+1)
    v-grid fields  (ny+1, nz, nx)

Restated pieces of the reference (input construction only, not the hot path):
    setup_simple_z          src/objects/domain_obj.f90:1743-1858 (Gal-Chen
                            coordinate with a flat top at the model lid)
    jacobian_u/_v/_w        src/objects/domain_obj.f90:1916-1931
    advection_dz            src/objects/domain_obj.f90:1960-1962
    calc_w / calc_divergence src/physics/wind.f90:166-262 (advect_density off)
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

F32 = np.float32

HYDROMETEORS = ("qc", "qr", "qi", "qs", "qg")
NUMBERS = {"nc": "qc", "nr": "qr", "ni": "qi", "ns": "qs", "ng": "qg"}
ALL12 = ("qv", "qc", "qr", "qi", "qs", "qg", "nr", "ni", "ns", "ng", "nc", "theta")


@dataclass
class Case:
    nx: int
    ny: int
    nz: int
    dx: float
    dz_levels: np.ndarray
    terrain: np.ndarray            # (ny, nx)
    u: np.ndarray                  # (ny, nz, nx+1)
    v: np.ndarray                  # (ny+1, nz, nx)
    w: np.ndarray                  # (ny, nz, nx)
    density: np.ndarray
    jacobian: np.ndarray
    jacobian_u: np.ndarray
    jacobian_v: np.ndarray
    jacobian_w: np.ndarray
    advection_dz: np.ndarray
    z: np.ndarray                  # cell-centre height (m)
    species: dict = field(default_factory=dict)   # name -> (ny, nz, nx)
    dt: float = 20.0
    # simple-microphysics inputs (add_mp_fields), (ny, nz, nx)
    pressure: np.ndarray | None = None
    exner: np.ndarray | None = None
    dz_mass: np.ndarray | None = None

    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    def copy(self) -> "Case":
        c = Case(**{k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self.__dict__.items()
                    if k != "species"})
        c.species = {k: v.copy() for k, v in self.species.items()}
        return c


# ---------------------------------------------------------------- terrain
def gaussian_ridge(nx: int, ny: int, dx: float, height: float, half_width: float) -> np.ndarray:
    """Gaussian hill of the given height and half-width, centred."""
    x = (np.arange(nx) - (nx - 1) / 2.0) * dx
    y = (np.arange(ny) - (ny - 1) / 2.0) * dx
    r2 = x[None, :] ** 2 + y[:, None] ** 2
    return (height * np.exp(-r2 / half_width ** 2)).astype(F32)


def fractal_terrain(nx: int, ny: int, dx: float, rms: float, hmax: float, rng: np.random.Generator,
                    slope: float = 3.0) -> np.ndarray:
    """Random-phase power-law terrain: spectrum ~ |k|^-slope, std = rms,
    shifted to a zero minimum and clipped at hmax."""
    kx = np.fft.rfftfreq(nx, d=dx)
    ky = np.fft.fftfreq(ny, d=dx)
    kk = np.sqrt(kx[None, :] ** 2 + ky[:, None] ** 2)
    kk[0, 0] = np.inf
    amp = kk ** (-slope / 2.0)
    phase = rng.uniform(0, 2 * np.pi, size=amp.shape)
    spec = amp * np.exp(1j * phase)
    h = np.fft.irfft2(spec, s=(ny, nx))
    h = (h - h.mean()) / (h.std() + 1e-30) * rms
    h = h - h.min()
    return np.minimum(h, hmax).astype(F32)


# ------------------------------------------------------- vertical grid / jacobians
def vertical_grid(terrain: np.ndarray, dz_levels: np.ndarray, nx: int, ny: int):
    """Gal-Chen terrain-following levels (setup_simple_z with the flat level
    at the model top) and the staggered jacobians of
    initialize_core_variables."""
    nz = len(dz_levels)
    dz = np.asarray(dz_levels, dtype=F32)
    H = F32(dz.sum())
    jac1 = ((H - terrain) / H).astype(F32)                          # (ny, nx)
    jac = np.empty((ny, nz, nx), F32)
    dzi = np.empty((ny, nz, nx), F32)
    for k in range(nz):
        dzi[:, k, :] = dz[k] * jac1
        jac[:, k, :] = dzi[:, k, :] / dz[k]
    # cell-centre height
    z = np.empty((ny, nz, nx), F32)
    zc = terrain + dzi[:, 0, :] / F32(2)
    z[:, 0, :] = zc
    for k in range(1, nz):
        zc = zc + (dz[k] / 2 * jac[:, k, :] + dz[k - 1] / 2 * jac[:, k - 1, :])
        z[:, k, :] = zc
    # jacobian_u: (ny, nz, nx+1), edges copy, interior average
    ju = np.empty((ny, nz, nx + 1), F32)
    ju[:, :, 0] = jac[:, :, 0]
    ju[:, :, nx] = jac[:, :, nx - 1]
    ju[:, :, 1:nx] = (jac[:, :, 1:] + jac[:, :, :-1]) / F32(2)
    jv = np.empty((ny + 1, nz, nx), F32)
    jv[0] = jac[0]
    jv[ny] = jac[ny - 1]
    jv[1:ny] = (jac[1:] + jac[:-1]) / F32(2)
    jw = np.empty((ny, nz, nx), F32)
    jw[:, nz - 1, :] = jac[:, nz - 1, :]
    jw[:, :nz - 1, :] = (dzi[:, :-1, :] * jac[:, :-1, :] + dzi[:, 1:, :] * jac[:, 1:, :]) / (dzi[:, :-1, :] + dzi[:, 1:, :])
    adz = np.empty((ny, nz, nx), F32)
    adz[:] = dz[None, :, None]
    return jac, ju, jv, jw, adz, z


def calc_w(u: np.ndarray, v: np.ndarray, ju: np.ndarray, jv: np.ndarray, jw: np.ndarray,
           adz: np.ndarray, dx: float) -> np.ndarray:
    """w from discrete continuity (calc_w with advect_density off) so that the
    Courant fluxes are divergence free cell by cell."""
    ny, nz, nxp = u.shape
    nx = nxp - 1
    um = u * ju
    vm = v * jv
    div = ((um[:, :, 1:] - um[:, :, :-1]) + (vm[1:] - vm[:-1])) / F32(dx)
    w = np.zeros((ny, nz, nx), F32)
    w[:, 0, :] = (F32(0) - div[:, 0, :] * adz[:, 0, :]) / jw[:, 0, :]
    for k in range(1, nz):
        w[:, k, :] = (w[:, k - 1, :] * jw[:, k - 1, :] - div[:, k, :] * adz[:, k, :]) / jw[:, k, :]
    return w.astype(F32)


def mountain_wave(terrain: np.ndarray, dx: float, z: np.ndarray, U: float, N: float):
    """Analytic hydrostatic linear mountain-wave perturbation (u', v') of a
    uniform westerly U over the terrain, evaluated at the cell-centre heights
    above the surface (linear theory as in linear_winds.f90, restated)."""
    ny, nx = terrain.shape
    h_hat = np.fft.fft2(terrain)
    k = 2 * np.pi * np.fft.fftfreq(nx, d=dx)[None, :]
    l = 2 * np.pi * np.fft.fftfreq(ny, d=dx)[:, None]
    kh2 = k ** 2 + l ** 2
    kh2[0, 0] = 1.0
    with np.errstate(divide="ignore", invalid="ignore"):
        m = np.where(np.abs(k) > 0, np.sign(U * k) * N * np.sqrt(kh2) / np.abs(U * k + 1e-30), 0.0)
    m = np.clip(m, -2 * np.pi / 500.0, 2 * np.pi / 500.0)
    nz = z.shape[1]
    up = np.empty((ny, nz, nx), F32)
    vp = np.empty((ny, nz, nx), F32)
    zagl = z - terrain[:, None, :]
    for kz in range(nz):
        zz = float(np.median(zagl[:, kz, :]))
        w_hat = 1j * U * k * h_hat * np.exp(1j * m * zz)
        u_hat = -k * m * w_hat / kh2
        v_hat = -l * m * w_hat / kh2
        up[:, kz, :] = np.real(np.fft.ifft2(u_hat))
        vp[:, kz, :] = np.real(np.fft.ifft2(v_hat))
    scale = max(1.0, float(np.abs(up).max()) / (0.5 * abs(U)))
    return up / scale, vp / scale


def smooth_field(shape, rng: np.random.Generator, coarse: int = 8) -> np.ndarray:
    """Spatially correlated noise: coarse normal noise repeated up to the grid."""
    ny, nz, nx = shape
    cz = max(1, coarse // 2)
    g = rng.standard_normal((ny // coarse + 2, nz // cz + 2, nx // coarse + 2)).astype(F32)
    g = np.repeat(np.repeat(np.repeat(g, coarse, 0), cz, 1), coarse, 2)
    oy, oz, ox = rng.integers(0, coarse), rng.integers(0, cz), rng.integers(0, coarse)
    return g[oy:oy + ny, oz:oz + nz, ox:ox + nx]


def correlated_noise(shape, rng: np.random.Generator, L: int = 8, Lz: int = 4) -> np.ndarray:
    """Smooth unit-variance noise: normal noise on a grid L cells apart (Lz
    levels apart), interpolated trilinearly to the full grid.  Used for the
    seeded wind perturbations: cell-to-cell (white) wind noise makes the flow
    strongly convergent from one cell to the next, and the reference scheme
    itself then grows without bound within tens of steps."""
    from scipy.ndimage import zoom
    ny, nz, nx = shape
    c = rng.standard_normal((ny // L + 3, nz // Lz + 3, nx // L + 3))
    f = zoom(c, (L, Lz, L), order=1)
    oy, oz, ox = (int(rng.integers(0, L)), int(rng.integers(0, Lz)), int(rng.integers(0, L)))
    f = f[oy:oy + ny, oz:oz + nz, ox:ox + nx]
    return ((f - f.mean()) / (f.std() + 1e-30)).astype(F32)


def hydrometeor(shape, rng, zero_frac=0.7, median=1e-4, sigma=1.0) -> np.ndarray:
    """Lognormal mixing ratio with an exact-zero fraction, zeros clustered."""
    s = smooth_field(shape, rng)
    thr = np.quantile(s, zero_frac)
    vals = (median * np.exp(sigma * rng.standard_normal(shape))).astype(F32)
    return np.where(s > thr, vals, F32(0)).astype(F32)


def make_species(names, z, rng, qv_noise=0.01, N=0.01):
    shape = z.shape
    out = {}
    masses = {}
    for nm in names:
        if nm == "qv":
            out[nm] = (0.010 * np.exp(-z / 2500.0) * (1 + qv_noise * rng.standard_normal(shape))).astype(F32)
        elif nm == "theta":
            out[nm] = (300.0 * np.exp(N * N * z / 9.81)).astype(F32)
        elif nm in HYDROMETEORS:
            masses[nm] = hydrometeor(shape, rng)
            out[nm] = masses[nm]
    for nm in names:
        if nm in NUMBERS:
            mass = masses.get(NUMBERS[nm])
            if mass is None:
                mass = hydrometeor(shape, rng)
            num = (1e5 * np.exp(1.0 * rng.standard_normal(shape))).astype(F32)
            out[nm] = np.where(mass > 0, num, F32(0)).astype(F32)
    return {nm: out[nm] for nm in names}


def build_case(nx, ny, nz, dx, dz_levels, terrain, U, V=0.0, mountain_N=None, wind_noise=0.0,
               species=("qv",), seed=0, dt=20.0, qv_noise=0.01) -> Case:
    rng = np.random.default_rng(seed)
    dz_levels = np.asarray(dz_levels, F32)
    if float(terrain.max()) >= float(dz_levels.sum()):
        raise ValueError("terrain reaches the model lid: the terrain-following jacobian would be <= 0")
    jac, ju, jv, jw, adz, z = vertical_grid(terrain, dz_levels, nx, ny)
    u = np.full((ny, nz, nx + 1), U, F32)
    v = np.full((ny + 1, nz, nx), V, F32)
    if mountain_N is not None:
        up, vp = mountain_wave(terrain, dx, z, U, mountain_N)
        u[:, :, 1:nx] += (up[:, :, 1:] + up[:, :, :-1]) / 2
        v[1:ny] += (vp[1:] + vp[:-1]) / 2
    if wind_noise > 0:
        u += (wind_noise * abs(U) * correlated_noise(u.shape, rng)).astype(F32)
        v += (wind_noise * abs(U) * correlated_noise(v.shape, rng)).astype(F32)
    w = calc_w(u, v, ju, jv, jw, adz, dx)
    density = (1.225 * np.exp(-z / 8500.0)).astype(F32)
    sp = make_species(species, z, rng, qv_noise=qv_noise)
    return Case(nx=nx, ny=ny, nz=nz, dx=float(dx), dz_levels=dz_levels, terrain=terrain, u=u, v=v, w=w,
                density=density, jacobian=jac, jacobian_u=ju, jacobian_v=jv, jacobian_w=jw,
                advection_dz=adz, z=z, species=sp, dt=float(dt))


# ------------------------------------------------------------- workloads
def config1(seed: int = 0, nx: int = 128, ny: int = 128, nz: int = 20) -> Case:
    """Plain MPDATA single domain: 128x128x20, dx 4 km, Gaussian ridge 1500 m
    (half-width 20 km), u = 10 m/s, v = 0, uniform 500 m levels, dt 20 s,
    one tracer qv."""
    dx = 4000.0
    terrain = gaussian_ridge(nx, ny, dx, 1500.0, 20000.0)
    return build_case(nx, ny, nz, dx, [500.0] * nz, terrain, U=10.0, species=("qv",), seed=seed, dt=20.0)


def config2(seed: int = 0, nx: int = 512, ny: int = 512, nz: int = 40) -> Case:
    """Full-species single domain: 512x512x40, dx 1 km, fractal terrain (RMS
    600 m, max 3000 m), 15 m/s westerly + linear mountain wave (N = 0.01/s)
    + 5 % noise, 12 advected fields, dt 4 s."""
    rng = np.random.default_rng(seed + 1000)
    dx = 1000.0
    terrain = fractal_terrain(nx, ny, dx, 600.0, 3000.0, rng)
    dzl = max(500.0, 20000.0 / nz)      # 500 m levels at nz=40; the lid stays at >= 20 km for small nz
    return build_case(nx, ny, nz, dx, [dzl] * nz, terrain, U=15.0, mountain_N=0.01, wind_noise=0.05,
                      species=ALL12, seed=seed, dt=4.0)


def ensemble_member(seed: int, nx: int, ny: int, nz: int) -> Case:
    """One member of the uneven ensemble: config-1-style ridge and winds on
    its own grid, with the 12-field state drawn from the config-2
    distributions."""
    rng = np.random.default_rng(seed)
    dx = 4000.0
    h = float(rng.uniform(800.0, 2000.0))
    terrain = gaussian_ridge(nx, ny, dx, h, 20000.0)
    return build_case(nx, ny, nz, dx, [500.0] * nz, terrain, U=float(rng.uniform(8.0, 12.0)),
                      species=ALL12, seed=seed, dt=20.0)


def ensemble_shapes(n: int = 64, seed: int = 0):
    """nx, ny ~ U[64,384], nz ~ U[20,50] for n members."""
    rng = np.random.default_rng(seed)
    return [(int(rng.integers(64, 385)), int(rng.integers(64, 385)), int(rng.integers(20, 51))) for _ in range(n)]


def config5(seed: int = 0, nx: int = 2048, ny: int = 2048, nz: int = 60) -> Case:
    """Large single domain: 2048x2048x60, dx 250 m, fractal terrain up to
    4000 m, 12 fields, dt 1 s."""
    rng = np.random.default_rng(seed + 5000)
    dx = 250.0
    terrain = fractal_terrain(nx, ny, dx, 800.0, 4000.0, rng)
    return build_case(nx, ny, nz, dx, [350.0] * nz, terrain, U=15.0, mountain_N=0.01, wind_noise=0.05,
                      species=ALL12, seed=seed, dt=1.0)


def periodic_y_case(ny: int = 100, nx: int = 3, nz: int = 3, cfl: float = 0.25, step: bool = True) -> Case:
    """The reference's own MPDATA test setup (src/tests/test_mpdata.f90:57-105):
    nx=3, ny=100, nz=3, a step function 1 -> 2 along y, y Courant 0.25, unit
    density, dz and jacobians.  The caller wraps rows 0 and ny-1 after every
    step to make it periodic."""
    dz_levels = np.ones(nz, F32)
    jac = np.ones((ny, nz, nx), F32)
    q = np.ones((ny, nz, nx), F32)
    if step:
        q[ny // 2:, :, :] = 2.0          # i > ny/2 (1-based)  ->  rows ny/2 .. ny-1
    else:
        rows = np.arange(1, ny + 1, dtype=F32)
        q[:] = (np.sin(rows / F32(ny - 2) * F32(2 * 3.141592)) + 1)[:, None, None]
    q[0] = q[ny - 2]
    q[ny - 1] = q[1]
    case = Case(nx=nx, ny=ny, nz=nz, dx=1.0, dz_levels=dz_levels, terrain=np.zeros((ny, nx), F32),
                u=np.zeros((ny, nz, nx + 1), F32), v=np.full((ny + 1, nz, nx), cfl, F32),
                w=np.zeros((ny, nz, nx), F32), density=np.ones((ny, nz, nx), F32), jacobian=jac,
                jacobian_u=np.ones((ny, nz, nx + 1), F32), jacobian_v=np.ones((ny + 1, nz, nx), F32),
                jacobian_w=np.ones((ny, nz, nx), F32), advection_dz=np.ones((ny, nz, nx), F32),
                z=np.zeros((ny, nz, nx), F32), species={"qv": q}, dt=1.0)
    return case


# ------------------------------------------------- on-device generation
def device_member(nx: int, ny: int, nz: int, seed: int, device: int = 0, dx: float = 4000.0,
                  dz: float = 500.0, species=ALL12, terrain_kind: str = "ridge", U: float | None = None,
                  noise: float = 0.02, dt: float = 20.0, rms: float = 800.0, hmax: float = 4000.0):
    """A config-1-style domain generated directly in GPU memory with torch
    (for served requests, whose inputs must appear in milliseconds, and for
    domains too large to build on the host): a Gaussian ridge (terrain_kind=
    "ridge") or random-phase power-law terrain of the given RMS clipped at
    hmax (terrain_kind="fractal"), Gal-Chen jacobians, uniform westerly (U, or a
    seeded 8..12 m/s) with seeded relative noise, w from discrete continuity,
    qv/theta profiles and clustered lognormal hydrometeors with ~70 % zeros.
    Returns (dict of float32 CUDA tensors in the Fortran layout of Case, dt)."""
    import torch
    g = torch.Generator(device=f"cuda:{device}")
    g.manual_seed(int(seed))
    dev = torch.device("cuda", device)
    f32 = torch.float32
    r = lambda *s: torch.rand(*s, generator=g, device=dev, dtype=f32)
    n = lambda *s: torch.randn(*s, generator=g, device=dev, dtype=f32)
    x = (torch.arange(nx, device=dev, dtype=f32) - (nx - 1) / 2.0) * dx
    y = (torch.arange(ny, device=dev, dtype=f32) - (ny - 1) / 2.0) * dx
    h = float(800.0 + 1200.0 * r(1).item())
    if terrain_kind == "fractal":
        kx = torch.fft.rfftfreq(nx, d=dx, device=dev)
        ky = torch.fft.fftfreq(ny, d=dx, device=dev)
        kk = torch.sqrt(kx[None, :] ** 2 + ky[:, None] ** 2)
        kk[0, 0] = float("inf")
        phase = 2 * torch.pi * torch.rand(kk.shape, generator=g, device=dev, dtype=torch.float64)
        spec = torch.polar(kk.double() ** -1.5, phase)
        t = torch.fft.irfft2(spec, s=(ny, nx))
        t = (t - t.mean()) / (t.std() + 1e-30) * rms
        terrain = torch.clamp(t - t.min(), max=hmax).to(f32)
        del kk, phase, spec, t
    else:
        terrain = h * torch.exp(-(x[None, :] ** 2 + y[:, None] ** 2) / 20000.0 ** 2)
    H = dz * nz
    if float(terrain.max()) >= H:
        raise ValueError("terrain reaches the model lid")
    jac1 = (H - terrain) / H
    jac = jac1[:, None, :].expand(ny, nz, nx).contiguous()
    dzi = dz * jac
    ju = torch.empty(ny, nz, nx + 1, device=dev, dtype=f32)
    ju[:, :, 0] = jac[:, :, 0]
    ju[:, :, nx] = jac[:, :, nx - 1]
    ju[:, :, 1:nx] = (jac[:, :, 1:] + jac[:, :, :-1]) / 2
    jv = torch.empty(ny + 1, nz, nx, device=dev, dtype=f32)
    jv[0] = jac[0]
    jv[ny] = jac[ny - 1]
    jv[1:ny] = (jac[1:] + jac[:-1]) / 2
    jw = torch.empty(ny, nz, nx, device=dev, dtype=f32)
    jw[:, nz - 1] = jac[:, nz - 1]
    jw[:, :nz - 1] = (dzi[:, :-1] * jac[:, :-1] + dzi[:, 1:] * jac[:, 1:]) / (dzi[:, :-1] + dzi[:, 1:])
    adz = torch.full((ny, nz, nx), dz, device=dev, dtype=f32)
    U = float(8.0 + 4.0 * r(1).item()) if U is None else float(U)

    def smooth(*shape, L=8, Lz=4):
        # unit-variance noise interpolated trilinearly from a grid L cells apart
        sy, sz, sx = shape
        c = n(1, 1, sy // L + 3, sz // Lz + 3, sx // L + 3)
        f = torch.nn.functional.interpolate(c, scale_factor=(L, Lz, L), mode="trilinear", align_corners=False)
        f = f[0, 0, :sy, :sz, :sx]
        return (f - f.mean()) / (f.std() + 1e-30)

    u = U + noise * U * smooth(ny, nz, nx + 1)
    v = noise * U * smooth(ny + 1, nz, nx)
    div = ((u * ju)[:, :, 1:] - (u * ju)[:, :, :-1] + (v * jv)[1:] - (v * jv)[:-1]) / dx
    w = torch.empty(ny, nz, nx, device=dev, dtype=f32)
    w[:, 0] = (0 - div[:, 0] * adz[:, 0]) / jw[:, 0]
    for k in range(1, nz):
        w[:, k] = (w[:, k - 1] * jw[:, k - 1] - div[:, k] * adz[:, k]) / jw[:, k]
    zc = terrain[:, None, :] + torch.cumsum(dzi, dim=1) - dzi / 2
    rho = 1.225 * torch.exp(-zc / 8500.0)

    def clustered(frac=0.7, median=1e-4):
        c = n(ny // 8 + 2, nz // 4 + 2, nx // 8 + 2)
        c = c.repeat_interleave(8, 0).repeat_interleave(4, 1).repeat_interleave(8, 2)[:ny, :nz, :nx]
        thr = torch.quantile(c.reshape(-1)[:: max(1, c.numel() // 100000)], frac)
        return torch.where(c > thr, median * torch.exp(n(ny, nz, nx)), torch.zeros((), device=dev))

    out = {"u": u, "v": v, "w": w, "density": rho, "jacobian": jac, "jacobian_u": ju, "jacobian_v": jv,
           "jacobian_w": jw, "advection_dz": adz}
    masses = {}
    sp = {}
    for nm in species:
        if nm == "qv":
            sp[nm] = 0.010 * torch.exp(-zc / 2500.0) * (1 + 0.01 * n(ny, nz, nx))
        elif nm == "theta":
            sp[nm] = 300.0 * torch.exp(1e-4 * zc / 9.81)
        elif nm in HYDROMETEORS:
            masses[nm] = clustered()
            sp[nm] = masses[nm]
    for nm in species:
        if nm in NUMBERS:
            m = masses.get(NUMBERS[nm])
            if m is None:
                m = clustered()
            sp[nm] = torch.where(m > 0, 1e5 * torch.exp(n(ny, nz, nx)), torch.zeros((), device=dev))
    out["species"] = {nm: sp[nm].to(f32).contiguous() for nm in species}
    for k in list(out):
        if k != "species":
            out[k] = out[k].to(f32).contiguous()
    return out, float(dt)


def device_config5(seed: int = 0, nx: int = 2048, ny: int = 2048, nz: int = 60, device: int = 0):
    """The large single domain (2048x2048x60, dx 250 m, fractal terrain up to
    4000 m, 12 fields, dt 1 s) generated on the device: building it on the
    host would take minutes and tens of GB of host memory."""
    return device_member(nx, ny, nz, seed, device=device, dx=250.0, dz=350.0, terrain_kind="fractal", U=15.0,
                         noise=0.05, dt=1.0, rms=800.0, hmax=4000.0)


def add_mp_fields(case: Case, moist: float = 1.5, seed: int = 0) -> Case:
    """Give a case the fields the simple microphysics reads: hydrostatic
    pressure from the cell heights (scale height 8 km, 1013.25 hPa at sea
    level), the exner function (p/1000 hPa)^(R/cp), dz_mass = the physical
    layer thickness (advection_dz * jacobian), and qv scaled by `moist` so
    some layers are supersaturated.  Rain and snow need qr/qs among the
    species (config 2 and the ensemble members carry all 12)."""
    z = case.z.astype(np.float64)
    p = 101325.0 * np.exp(-z / 8000.0)
    case.pressure = p.astype(F32)
    case.exner = ((p / 100000.0) ** (287.058 / 1004.5)).astype(F32)
    case.dz_mass = (case.advection_dz * case.jacobian).astype(F32)
    if "qv" in case.species:
        case.species["qv"] = (case.species["qv"] * F32(moist)).astype(F32)
    return case
