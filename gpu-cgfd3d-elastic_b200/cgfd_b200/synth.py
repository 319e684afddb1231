"""Seeded synthetic inputs in the reference's formats.

No public dataset is involved: the workloads are curvilinear grids with a Gaussian hill plus
random relief, layered media with an optional von Karman perturbation, random double-couple
moment sources and surface station grids, following the configurations the benchmark is
quoted on (100x100x60 at 100 m; 480x480x240 at 50 m; ...).
"""
import ctypes as C

import numpy as np

from .abi import (CGFD_MEDIUM_ACOUSTIC_ISO, CGFD_MEDIUM_ELASTIC_ISO, CGFD_MEDIUM_ELASTIC_VTI, CGFD_MEDIUM_ELASTIC_ANISO, WAVELETS,
                  CGFD_MEDIUM_VISCO_ISO,
                  Problem, Sources, Stations, lib, ref_shape, ProblemDesc)

LAYERS_3 = [(4000.0, 2300.0, 2500.0), (5500.0, 3200.0, 2700.0), (6500.0, 3750.0, 2900.0)]
INTERFACES_3 = [-1500.0, -3500.0]


def _gauss_filter_2d(noise, corr_pts):
    """Isotropic Gaussian filtering by FFT, correlation length in grid points."""
    ny, nx = noise.shape
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.fftfreq(nx)[None, :]
    k2 = kx * kx + ky * ky
    filt = np.exp(-(np.pi * corr_pts) ** 2 * k2)
    return np.real(np.fft.ifft2(np.fft.fft2(noise) * filt))


def topography(ni, nj, dh, amp=300.0, sigma=1500.0, relief_std=20.0, relief_corr=500.0, seed=0):
    """Surface height [nj, ni]: centred Gaussian hill + Gaussian-filtered white noise."""
    rng = np.random.default_rng(seed)
    x = (np.arange(ni) - (ni - 1) / 2.0) * dh
    y = (np.arange(nj) - (nj - 1) / 2.0) * dh
    X, Y = np.meshgrid(x, y)
    hill = amp * np.exp(-(X * X + Y * Y) / (2.0 * sigma * sigma))
    noise = _gauss_filter_2d(rng.standard_normal((nj, ni)), relief_corr / dh)
    noise *= relief_std / max(noise.std(), 1e-30)
    return hill + noise


def curvilinear_grid(ni, nj, nk, dh, depth=None, stretch=0.3, **topo_kw):
    """Coordinates [3, nz, ny, nx] (reference layout, ghosts filled by linear extrapolation).

    x, y uniform with spacing dh; z from a flat bottom at -depth to the topography, with
    s(u) = u + stretch*u*(1-u) so that cells are finer towards the surface.
    """
    depth = (nk - 1) * dh if depth is None else depth
    topo = topography(ni, nj, dh, **topo_kw)
    u = np.linspace(0.0, 1.0, nk)
    s = u + stretch * u * (1.0 - u)
    zb = -depth
    coord = np.zeros((3,) + ref_shape(ni, nj, nk), np.float32)
    x = np.arange(ni) * dh
    y = np.arange(nj) * dh
    coord[0, 3:-3, 3:-3, 3:-3] = x[None, None, :]
    coord[1, 3:-3, 3:-3, 3:-3] = y[None, :, None]
    coord[2, 3:-3, 3:-3, 3:-3] = (zb + (topo[None, :, :] - zb) * s[:, None, None]).astype(np.float32)
    fill_ghosts(coord)
    return coord


def fill_ghosts(v4d):
    ncmp, nz, ny, nx = v4d.shape
    rc = lib().cgfd_fill_ghosts(nx - 6, ny - 6, nz - 6, ncmp, v4d.ctypes.data)
    assert rc == 0


def metrics(coord):
    """FP64 metrics [10, nz, ny, nx] via cgfd_metric_calc."""
    _, nz, ny, nx = coord.shape
    out = np.zeros((10, nz, ny, nx), np.float32)
    c = np.ascontiguousarray(coord, np.float32)
    rc = lib().cgfd_metric_calc(nx - 6, ny - 6, nz - 6, c.ctypes.data, out.ctypes.data)
    assert rc == 0
    return out


def metrics_gpu(coord, device=0):
    """FP64 metrics [10, nz, ny, nx] computed on the GPU via cgfd_metric_calc_gpu."""
    _, nz, ny, nx = coord.shape
    out = np.zeros((10, nz, ny, nx), np.float32)
    c = np.ascontiguousarray(coord, np.float32)
    rc = lib().cgfd_metric_calc_gpu(int(device), nx - 6, ny - 6, nz - 6, c.ctypes.data, out.ctypes.data)
    if rc != 0:
        raise RuntimeError(lib().cgfd_last_error().decode())
    return out


def von_karman(shape, dh, corr=1000.0, hurst=0.3, std=0.05, seed=1):
    """Seeded 3-D von Karman random field (zero mean, given std) on `shape` (nk, nj, ni)."""
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal(shape).astype(np.float32)
    try:
        import scipy.fft as sfft
        F = sfft.rfftn(noise, workers=-1)
    except Exception:  # numpy fallback for input generation only
        F = np.fft.rfftn(noise)
    k = [np.fft.fftfreq(n, d=dh) * 2 * np.pi for n in shape[:-1]] + [np.fft.rfftfreq(shape[-1], d=dh) * 2 * np.pi]
    k2 = (k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2 + k[2][None, None, :] ** 2).astype(np.float32)
    # power spectrum ~ (1 + k^2 a^2)^-(H + 3/2); amplitude filter is its square root
    F *= (1.0 + k2 * corr * corr) ** (-(hurst + 1.5) / 2.0)
    try:
        import scipy.fft as sfft
        f = sfft.irfftn(F, s=shape, workers=-1)
    except Exception:
        f = np.fft.irfftn(F, s=shape)
    f = f.astype(np.float32)
    f -= f.mean()
    f *= std / max(float(f.std()), 1e-30)
    return f


def layered_iso(coord, layers=LAYERS_3, interfaces=INTERFACES_3, perturb=None):
    """Elastic iso medium [3, nz, ny, nx] (rho, lambda, mu) from flat layers by depth z,
    optionally scaled by (1 + perturb) on vp, vs, rho."""
    z = coord[2]
    vp = np.full(z.shape, layers[-1][0], np.float32)
    vs = np.full(z.shape, layers[-1][1], np.float32)
    rho = np.full(z.shape, layers[-1][2], np.float32)
    for n in range(len(interfaces) - 1, -1, -1):
        m = z > interfaces[n]
        vp[m], vs[m], rho[m] = layers[n]
    if perturb is not None:
        sl = (slice(3, -3),) * 3
        f = 1.0 + perturb
        vp[sl] *= f
        vs[sl] *= f
        rho[sl] *= f
    med = np.zeros((3,) + z.shape, np.float32)
    med[0] = rho
    med[1] = rho * (vp * vp - 2.0 * vs * vs)
    med[2] = rho * vs * vs
    return med


def layered_ac(coord, layers=LAYERS_3, interfaces=INTERFACES_3):
    """Acoustic iso medium [2, nz, ny, nx] (rho, kappa = rho vp^2) from the flat layers of
    layered_iso (their vp and rho)."""
    iso = layered_iso(coord, layers, interfaces)
    med = np.zeros((2,) + iso.shape[1:], np.float32)
    med[0] = iso[0]
    med[1] = iso[1] + 2.0 * iso[2]  # lambda + 2 mu = rho vp^2
    return med


def layer_model(coord, seed=5, layers=LAYERS_3, depths=(-1500.0, -3500.0), relief=150.0, grad=True):
    """A layered elastic-isotropic model (formats.LayerModel) over the grid's horizontal extent:
    a free top interface above the topography, then undulating interfaces around the given
    depths (seeded sinusoidal relief), each layer with vp / vs / rho of `layers` and, with
    `grad`, a small depth gradient (power 1)."""
    from .formats import LayerModel
    rng = np.random.default_rng(seed)
    x, y = coord[0], coord[1]
    x0, x1 = float(x.min()) - 100.0, float(x.max()) + 100.0
    y0, y1 = float(y.min()) - 100.0, float(y.max()) + 100.0
    nx, ny = 41, 37
    dx, dy = (x1 - x0) / (nx - 1), (y1 - y0) / (ny - 1)
    X, Y = np.meshgrid(x0 + dx * np.arange(nx), y0 + dy * np.arange(ny))
    top = np.full((ny, nx), float(coord[2].max()) + 1000.0)
    elev = [top]
    for d in depths:
        kx, ky, ph = rng.uniform(0.5, 2.0), rng.uniform(0.5, 2.0), rng.uniform(0, 6.3)
        elev.append(d + relief * np.sin(kx * 2 * np.pi * (X - x0) / (x1 - x0) + ph) *
                    np.cos(ky * 2 * np.pi * (Y - y0) / (y1 - y0)))
    ni = len(elev)
    f = {"elevation": np.stack(elev)}
    for q, name in enumerate(("vp", "vs", "rho")):
        vals = np.array([lay[q] for lay in layers], np.float32)
        f[name] = np.repeat(vals[:, None, None], ny, 1).repeat(nx, 2)
        f[name + "_grad"] = np.full((ni, ny, nx), (0.05 if grad else 0.0) * (q < 2), np.float32)
        f[name + "_pow"] = np.ones((ni, ny, nx), np.float32)
    return LayerModel(x0, y0, dx, dy, **f)


def bin_model(coord, seed=5, order=(2, 0, 1), spacing=(60.0, 90.0, 80.0), margin=300.0):
    """A binary model (formats.BinModel) over the grid's extent plus `margin`: vp, vs, rho
    rising smoothly with depth across the interfaces of INTERFACES_3 (below the speeds of the
    deepest of LAYERS_3), with a seeded lateral variation of 2%, sampled on a regular mesh whose file dimensions run along the grid axes `order`
    (default z fastest, then x, then y) with `spacing` per grid axis x, y, z; z decreasing from the
    top of the grid (origin at the top, negative spacing), as depth models are stored."""
    from .formats import BinModel
    rng = np.random.default_rng(seed)
    lo = [float(coord[a].min()) - margin for a in range(3)]
    hi = [float(coord[a].max()) + margin for a in range(3)]
    sp = [float(spacing[0]), float(spacing[1]), -float(spacing[2])]
    org = [lo[0], lo[1], hi[2]]
    n = [int(np.ceil((hi[a] - lo[a]) / abs(sp[a]))) + 1 for a in range(3)]
    ax = [org[a] + sp[a] * np.arange(n[a]) for a in range(3)]
    Z, Y, X = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")  # grid-axis order (z, y, x)
    # 0 above the first interface, 1 below the second; speeds stay below the deepest layer's
    t = 0.25 * (1 + np.tanh((-Z - 1500.0) / 300.0)) + 0.25 * (1 + np.tanh((-Z - 3500.0) / 300.0))
    vp = LAYERS_3[0][0] + t * (LAYERS_3[2][0] - LAYERS_3[0][0]) * 0.9
    vs = LAYERS_3[0][1] + t * (LAYERS_3[2][1] - LAYERS_3[0][1]) * 0.9
    rho = LAYERS_3[0][2] + t * (LAYERS_3[2][2] - LAYERS_3[0][2]) * 0.9
    k = rng.uniform(1.0, 3.0, 2) * 2 * np.pi / max(hi[0] - lo[0], 1.0)
    lat = 1.0 + 0.02 * np.sin(k[0] * X + rng.uniform(0, 6.3)) * np.cos(k[1] * Y + rng.uniform(0, 6.3))
    vols = [np.asarray(v * lat, np.float32) for v in (rho, vp, vs)]
    # file order: file dimension d runs along grid axis order[d], dimension 0 fastest
    perm = [2 - order[2], 2 - order[1], 2 - order[0]]  # numpy axes (z=0, y=1, x=2) of file dims 2, 1, 0
    vols = [np.ascontiguousarray(np.transpose(v, perm)) for v in vols]
    size = [n[order[d]] for d in range(3)]
    return BinModel(order, size, [sp[order[d]] for d in range(3)], [org[order[d]] for d in range(3)], *vols)


def grid_media(coord, seed=5, ngz=(3, 4, 3), depths=(-1200.0, -2400.0), relief=150.0, margin=300.0, type=21):
    """A grid model (formats.GridMedia) over the grid's extent plus `margin`: len(ngz) layers whose
    tops lie above the grid and undulate around `depths`, each layer given by ngz[l] >= 2 surfaces
    evenly spaced from its top down to the next layer's top (the last layer's down to 1.5 km below
    its top), so that a layer's last surface lies on the next layer's first, as the format asks;
    rho, vp, vs of LAYERS_3 per layer (other file types: the per-layer parameters of layer_media),
    the speeds and stiffnesses rising a few percent from a layer's top surface to its last one,
    with a seeded lateral variation."""
    from .formats import GridMedia, LAYER_TYPES
    rng = np.random.default_rng(seed)
    dx = dy = 100.0
    x0 = float(coord[0].min()) - margin
    y0 = float(coord[1].min()) - margin
    nx = int(np.ceil((float(coord[0].max()) + margin - x0) / dx)) + 1
    ny = int(np.ceil((float(coord[1].max()) + margin - y0) / dy)) + 1
    X, Y = np.meshgrid(x0 + dx * np.arange(nx), y0 + dy * np.arange(ny))
    tops = [float(coord[2].max()) + 200.0] + list(depths)
    def surface(z, n):
        k = rng.uniform(1.0, 3.0, 2) * 2 * np.pi / max(nx * dx, 1.0)
        return z + relief * np.sin(k[0] * X + rng.uniform(0, 6.3)) * np.cos(k[1] * Y + rng.uniform(0, 6.3)) * (n > 0)
    names = LAYER_TYPES[type][1]
    lm = layer_media(coord, type, seed=seed) if type != 21 else None
    surf = [np.asarray(surface(tops[l], l), np.float32) for l in range(len(ngz))]
    surf.append(surf[-1] - np.float32(1500.0))
    elev, par = [], []
    for l, ng in enumerate(ngz):
        top, bot = surf[l], surf[l + 1]
        vp, vs, rho = LAYERS_3[min(l, len(LAYERS_3) - 1)]
        base = [rho, vp, vs] if type == 21 else [float(v) for v in lm.param[:, 0, min(l, lm.param.shape[2] - 1), 0, 0]]
        for s in range(ng):
            f = s / max(ng - 1, 1)
            elev.append(bot if s == ng - 1 else top + (bot - top) * np.float32(f))
            lat = 1.0 + 0.01 * np.sin(X / 700.0 + l) * np.cos(Y / 900.0 + s)
            g = 1.0 + 0.04 * f
            par.append([b * g * lat if (nm == "rho" or nm[0] in "vc") else b + 0 * X
                        for b, nm in zip(base, names)])
    elev = np.asarray(elev, np.float32)
    param = np.asarray(par, np.float32).transpose(1, 0, 2, 3)
    return GridMedia(ngz, x0, y0, dx, dy, elev, param, type)


def layer_media(coord, type, seed=5, depths=(-1500.0, -3500.0), relief=150.0, grad=True):
    """A layer file of media type `type` (formats.LAYER_TYPES) over the grid's horizontal extent,
    with the interfaces of layer_model (a free top interface, undulating interfaces around the
    given depths) and seeded per-layer parameters: speeds of LAYERS_3 with Thomsen epsilon in
    [0, 0.2], delta in [-0.1, 0.1], gamma in [0, 0.15], PREM-style vph / vsh a few percent above
    vpv / vsv and eta near 1, stiffnesses from those (Cij files), and with `grad` a small depth
    gradient (power 1) on the speeds and the stiffnesses. The tilt (azimuth in [0, 360), dip in
    [10, 60] degrees) and the extra terms of the 21-Cij file are the same in every layer, so
    that no c_ij changes sign across an interface (the harmonic average of a c_ij that does is
    ill-conditioned)."""
    from .formats import LayerMedia, LAYER_TYPES
    base = layer_model(coord, seed=seed, depths=depths, relief=relief, grad=False)
    rng = np.random.default_rng(seed + 100)
    ni, ny, nx = base.elevation.shape
    names = LAYER_TYPES[type][1]
    az, dip = rng.uniform(0.0, 360.0), rng.uniform(10.0, 60.0)
    E0 = rng.normal(0.0, 0.02, (6, 6))
    E0 = (E0 + E0.T) / 2
    per = []  # per layer: parameter values
    for n in range(ni):
        vp, vs, rho = LAYERS_3[min(n, len(LAYERS_3) - 1)]
        eps, dlt, gam = rng.uniform(0.0, 0.2), rng.uniform(-0.1, 0.1), rng.uniform(0.0, 0.15)
        c33, c55 = rho * vp * vp, rho * vs * vs
        c11, c66 = c33 * (1 + 2 * eps), c55 * (1 + 2 * gam)
        c13 = np.sqrt(2 * dlt * c33 * (c33 - c55) + (c33 - c55) ** 2) - c55
        v = {"rho": rho, "vp": vp, "vs": vs, "vph": vp * 1.03, "vpv": vp, "vsh": vs * 1.04, "vsv": vs,
             "eta": rng.uniform(0.9, 1.0), "vp0": vp, "vs0": vs, "epsilon": eps, "delta": dlt, "gamma": gam,
             "azimuth": az, "dip": dip, "c11": c11, "c33": c33, "c55": c55, "c66": c66, "c13": c13}
        if type == 27:  # a rotated TI tensor with small extra terms
            C = np.zeros((6, 6))
            C[0, 0] = C[1, 1] = c11
            C[2, 2] = c33
            C[0, 1] = C[1, 0] = c11 - 2 * c66
            C[0, 2] = C[2, 0] = C[1, 2] = C[2, 1] = c13
            C[3, 3] = C[4, 4] = c55
            C[5, 5] = c66
            C = C + E0 * c55
            for a in range(6):
                for b in range(a, 6):
                    v["c%d%d" % (a + 1, b + 1)] = C[a, b]
        per.append(v)
    param = np.zeros((len(names), 3, ni, ny, nx), np.float32)
    for q, nm in enumerate(names):
        for n in range(ni):
            param[q, 0, n] = per[n][nm]
            speed_or_stiff = nm.startswith("v") or nm.startswith("c")
            param[q, 1, n] = (0.05 if nm.startswith("v") else 5e3) if (grad and speed_or_stiff) else 0.0
            param[q, 2, n] = 1.0
    return LayerMedia(type, base.x0, base.y0, base.dx, base.dy, base.elevation, param)


def thomsen_vti(coord, seed=2, layers=LAYERS_3, interfaces=INTERFACES_3):
    """VTI medium [6, ...] (rho, c11, c13, c33, c55, c66) from layered Thomsen parameters
    eps in [0, 0.2], delta in [-0.1, 0.1], gamma in [0, 0.15] (seeded per layer)."""
    rng = np.random.default_rng(seed)
    nl = len(layers)
    eps = rng.uniform(0.0, 0.2, nl)
    dlt = rng.uniform(-0.1, 0.1, nl)
    gam = rng.uniform(0.0, 0.15, nl)
    z = coord[2]
    lay = np.full(z.shape, nl - 1, np.int32)
    for n in range(len(interfaces) - 1, -1, -1):
        lay[z > interfaces[n]] = n
    out = np.zeros((6,) + z.shape, np.float32)
    for n, (vp, vs, rho) in enumerate(layers):
        c33 = rho * vp * vp
        c55 = rho * vs * vs
        c11 = c33 * (1 + 2 * eps[n])
        c66 = c55 * (1 + 2 * gam[n])
        c13 = np.sqrt(max((c33 - c55) * (c33 - c55) + 2 * dlt[n] * c33 * (c33 - c55), 1e-6)) - c55
        m = lay == n
        for c, v in enumerate([rho, c11, c13, c33, c55, c66]):
            out[c][m] = v
    return out


def _bond(R):
    """6x6 Bond matrix of rotation R (Voigt xx yy zz yz xz xy)."""
    M = np.zeros((6, 6))
    idx = [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]
    for I, (i, j) in enumerate(idx):
        for J, (k, l) in enumerate(idx):
            if J < 3:
                M[I, J] = R[i, k] * R[j, l]
            else:
                M[I, J] = R[i, k] * R[j, l] + R[i, l] * R[j, k]
    return M


def tilted_aniso(coord, seed=3, layers=LAYERS_3, interfaces=INTERFACES_3):
    """Full 21-Cij medium [22, ...] from Bond-rotated Thomsen TI layers (seeded tilt/azimuth)."""
    vti = thomsen_vti(coord, seed=seed, layers=layers, interfaces=interfaces)
    rng = np.random.default_rng(seed + 100)
    z = coord[2]
    nl = len(layers)
    lay = np.full(z.shape, nl - 1, np.int32)
    for n in range(len(interfaces) - 1, -1, -1):
        lay[z > interfaces[n]] = n
    out = np.zeros((22,) + z.shape, np.float32)
    for n in range(nl):
        m = lay == n
        if not m.any():
            continue
        p = np.argwhere(m)[0]
        rho, c11, c13, c33, c55, c66 = [float(vti[c][tuple(p)]) for c in range(6)]
        C6 = np.zeros((6, 6))
        c12 = c11 - 2 * c66
        C6[0, 0] = C6[1, 1] = c11
        C6[0, 1] = C6[1, 0] = c12
        C6[0, 2] = C6[2, 0] = C6[1, 2] = C6[2, 1] = c13
        C6[2, 2] = c33
        C6[3, 3] = C6[4, 4] = c55
        C6[5, 5] = c66
        tilt = np.deg2rad(rng.uniform(0, 45))
        azi = np.deg2rad(rng.uniform(0, 360))
        Ry = np.array([[np.cos(tilt), 0, np.sin(tilt)], [0, 1, 0], [-np.sin(tilt), 0, np.cos(tilt)]])
        Rz = np.array([[np.cos(azi), -np.sin(azi), 0], [np.sin(azi), np.cos(azi), 0], [0, 0, 1]])
        Mb = _bond(Rz @ Ry)
        Cr = Mb @ C6 @ Mb.T
        out[0][m] = rho
        q = 1
        for a in range(6):
            for b in range(a, 6):
                out[q][m] = Cr[a, b]
                q += 1
    return out


def column_depth_index(coord, i, j, depth):
    """Fractional depth index (counted down from the surface) at which z = surface - depth."""
    z = coord[2, 3:-3, j + 3, i + 3].astype(np.float64)
    target = z[-1] - depth
    nk = z.shape[0]
    kf = float(np.interp(target, z, np.arange(nk)))
    return (nk - 1) - kf


def random_dc(rng):
    return rng.uniform(0, 360), rng.uniform(0, 90), rng.uniform(-180, 180)


def dc_sources(coord, ni, nj, n, rng, depth_range=(2000.0, 2000.0), fc_range=(2.0, 2.0), m0=1e16,
               center=False, stf_length=None, dt=None):
    """Random double-couple sources given by strike/dip/rake + mu D A (mechanism_type 1),
    located by grid index with the depth flag, Ricker source time functions."""
    loc = np.zeros((n, 3), np.float32)
    cmp = np.zeros((n, 9), np.float32)
    coefs = np.zeros((n, 10), np.float32)
    tstart = np.zeros(n, np.float32)
    for s in range(n):
        if center:
            i, j = ni // 2, nj // 2
        else:
            i = int(rng.integers(ni // 4, 3 * ni // 4))
            j = int(rng.integers(nj // 4, 3 * nj // 4))
        dep = rng.uniform(*depth_range)
        loc[s] = (i, j, column_depth_index(coord, i, j, dep))
        strike, dip, rake = random_dc(rng)
        mu = 3.0e10
        area = m0 / mu
        cmp[s, 3:9] = (strike, dip, rake, mu, 1.0, area)
        fc = rng.uniform(*fc_range)
        coefs[s, 0], coefs[s, 1] = fc, 1.2 / fc
    return Sources(loc=loc, t_start=tstart, wavelet=np.full(n, WAVELETS["ricker"], np.int32),
                   wavelet_coefs=coefs, cmp=cmp, stf_given=0, stf_length=float(stf_length),
                   cmp_type=2, mechanism_type=1, loc_coord_type=0, loc_3dim=1)


def ac_sources(coord, ni, nj, n, rng, depth_range=(2000.0, 2000.0), fc_range=(2.0, 2.0), m0=1e16, center=False,
               stf_length=None, dt=None):
    """Sources of acoustic problems: a pressure term (moment components given directly, Mxx
    drives P; the others are set too and must stay without effect) and a random force
    (cmp_type 3), located by grid index with the depth flag, Ricker source time functions."""
    loc = np.zeros((n, 3), np.float32)
    cmp = np.zeros((n, 9), np.float32)
    coefs = np.zeros((n, 10), np.float32)
    tstart = np.zeros(n, np.float32)
    for s in range(n):
        if center:
            i, j = ni // 2, nj // 2
        else:
            i = int(rng.integers(ni // 4, 3 * ni // 4))
            j = int(rng.integers(nj // 4, 3 * nj // 4))
        dep = rng.uniform(*depth_range)
        loc[s] = (i, j, column_depth_index(coord, i, j, dep))
        f = rng.normal(size=3)
        cmp[s, 0:3] = (m0 * 1e-3) * f / np.linalg.norm(f)
        cmp[s, 3:9] = m0 * np.array([1.0, 0.7, 0.4, 0.3, -0.2, 0.1])
        fc = rng.uniform(*fc_range)
        coefs[s, 0], coefs[s, 1] = fc, 1.2 / fc
    return Sources(loc=loc, t_start=tstart, wavelet=np.full(n, WAVELETS["ricker"], np.int32),
                   wavelet_coefs=coefs, cmp=cmp, stf_given=0, stf_length=float(stf_length),
                   cmp_type=3, mechanism_type=0, loc_coord_type=0, loc_3dim=1)


def surface_stations(ni, nj, nx_sta, ny_sta, margin=0.15):
    """nx_sta*ny_sta stations on the surface (1-based grid index, depth flag, z = 0)."""
    xs = np.round(np.linspace(margin * (ni - 1), (1 - margin) * (ni - 1), nx_sta)) + 1
    ys = np.round(np.linspace(margin * (nj - 1), (1 - margin) * (nj - 1), ny_sta)) + 1
    X, Y = np.meshgrid(xs, ys)
    loc = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], 1).astype(np.float32)
    return Stations(loc=loc, flag_depth=np.ones(X.size, np.int32),
                    names=[f"sta{n:04d}" for n in range(X.size)])


def pml_all(n, alpha_max=3.0, beta_max=2.5, ref_vel=6500.0):
    f = {"num_layers": n, "alpha_max": alpha_max, "beta_max": beta_max, "ref_vel": ref_vel}
    return [[f, f], [f, f], [f, None]]


def dt_estimate(prob, cfl=1.3):
    d = prob.desc()
    out = C.c_double()
    rc = lib().cgfd_dt_estimate(C.byref(d), cfl, C.byref(out))
    assert rc == 0
    return out.value


def keep_three_digits(dt):
    return float(lib().cgfd_keep_three_digits(float(dt)))


def make_problem(ni, nj, nk, dh, nsteps, dt=None, medium="iso", npml=12, nsrc=1, sta_grid=(5, 5),
                 fc=2.0, seed=0, perturb_std=0.0, corr=1000.0, hurst=0.3, src_depth=(2000.0, 2000.0),
                 center_src=True, metric_fn=None, free_top=1, stf_length=None):
    """Build a seeded Problem of the benchmark family.

    medium: "iso" (3 flat layers, optional von Karman perturbation), "vti" (layered Thomsen),
    "aniso" (Bond-rotated tilted TI), "ac" (acoustic, the iso layers' vp and rho; sources with
    a force and an Mxx pressure term). dt=None -> keep_three_digits(0.9 * dtmax).
    """
    coord = curvilinear_grid(ni, nj, nk, dh, seed=seed)
    metric = metrics(coord) if metric_fn is None else metric_fn(coord)
    if medium in ("iso", "vis"):
        pert = None
        if perturb_std > 0:
            pert = von_karman((nk, nj, ni), dh, corr=corr, hurst=hurst, std=perturb_std, seed=seed + 1)
        med = layered_iso(coord, perturb=pert)
        mtype = CGFD_MEDIUM_ELASTIC_ISO
        vmax = float(np.sqrt((med[1] + 2 * med[2]) / np.maximum(med[0], 1e-9))[3:-3, 3:-3, 3:-3].max())
    elif medium == "vti":
        med = thomsen_vti(coord, seed=seed + 2)
        mtype = CGFD_MEDIUM_ELASTIC_VTI
        vmax = float(np.sqrt(np.maximum(med[1], med[3]) / np.maximum(med[0], 1e-9))[3:-3, 3:-3, 3:-3].max())
    elif medium == "aniso":
        med = tilted_aniso(coord, seed=seed + 3)
        mtype = CGFD_MEDIUM_ELASTIC_ANISO
        vmax = float(np.sqrt(np.maximum(np.maximum(med[1], med[7]), med[12]) / np.maximum(med[0], 1e-9))[3:-3, 3:-3, 3:-3].max())
    elif medium == "ac":
        med = layered_ac(coord)
        mtype = CGFD_MEDIUM_ACOUSTIC_ISO
        vmax = float(np.sqrt(med[1] / np.maximum(med[0], 1e-9))[3:-3, 3:-3, 3:-3].max())
    else:
        raise ValueError(medium)
    prob = Problem(ni=ni, nj=nj, nk=nk, medium_type=mtype, coord=coord, metric=metric, medium=med,
                   dt=1.0, nt_total=nsteps + 1, free_top=free_top)
    if npml:
        prob.pml = pml_all(npml, ref_vel=vmax)
        if not free_top:
            prob.pml[2][1] = prob.pml[2][0]
    if dt is None:
        dt = keep_three_digits(0.9 * dt_estimate(prob))
    prob.dt = float(dt)
    if medium == "vis":
        # visco-elastic: the iso layers with Qs = 20 + vs / 50 and Qp = 2 Qs, three GMB mechanisms
        # over 0.2-20 Hz with the moduli given at 2 Hz (the time step above is the elastic one;
        # the unrelaxed moduli are a few per cent stiffer, inside its 0.9 margin)
        vs = np.sqrt(med[2] / np.maximum(med[0], 1e-9))
        qs = np.round(20.0 + vs / 50.0).astype(np.float32)
        prob.medium = np.concatenate([med, (2.0 * qs)[None], qs[None]]).astype(np.float32)
        prob.medium_type = CGFD_MEDIUM_VISCO_ISO
        prob.visco = {"nmaxwell": 3, "fr": 2.0, "fmin": 0.2, "fmax": 20.0}
    rng = np.random.default_rng(seed + 7)
    if nsrc:
        mk = ac_sources if medium == "ac" else dc_sources
        prob.src = mk(coord, ni, nj, nsrc, rng, depth_range=src_depth, fc_range=(fc, fc) if np.isscalar(fc) else fc,
                      center=center_src, stf_length=stf_length if stf_length else (nsteps + 1) * dt)
    if sta_grid:
        prob.sta = surface_stations(ni, nj, *sta_grid)
    return prob
