"""Seeded synthetic landscapes with the shapes of the reference workloads.

No public dataset is involved: every mesh and field is generated here from a
seed.  Generators:

* ``planar_hex_mesh`` — jittered hexagonal lattice over a square, Delaunay
  triangulated (scipy/qhull), boundary vertices exactly on the square's edges.
* ``icosphere`` — icosahedron refined ``level`` times: N = 10*4**level + 2
  vertices on a sphere of radius R.
* ``fractal_field`` — k^-beta power-spectrum noise on a periodic grid, sampled
  bilinearly at the vertices.
* ``sh_field`` — random real spherical-harmonic field to degree ``lmax`` with
  per-degree power proportional to l^-beta, synthesised on a latitude grid by
  Legendre recursion plus an FFT in longitude, sampled bilinearly.
* ``belt_uplift`` — sum of Gaussian belts around random great circles.

The per-workload recipes (``planar_config``, ``sphere_config``,
``ensemble_member``, ``inversion_config``) return numpy arrays in the goSPL
``.npz`` convention (``v`` coordinates, ``c`` int32 cells, ``z`` elevation)
plus the forcing fields and parameters.
"""
import numpy as np

EARTH_RADIUS = 6371.0e3


# ----------------------------------------------------------------------------
# meshes
# ----------------------------------------------------------------------------
def planar_hex_mesh(n_target, side, seed, jitter=0.25):
    """Jittered hex lattice with ~n_target vertices over [0, side]^2."""
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    # hex cell area = sqrt(3)/2 s^2  ->  s from area per vertex
    s = np.sqrt(side * side / n_target / (np.sqrt(3.0) / 2.0))
    dy = s * np.sqrt(3.0) / 2.0
    nrow = int(np.floor(side / dy))
    pts = []
    for j in range(1, nrow + 1):
        y = j * dy
        if y > side - 0.5 * dy:
            break
        off = 0.5 * s if (j % 2) else 0.0
        x = np.arange(off + s, side - 0.5 * s, s)
        pts.append(np.stack([x, np.full_like(x, y)], axis=1))
    interior = np.concatenate(pts)
    # jitter inside a disk of radius jitter*s
    r = jitter * s * np.sqrt(rng.random(len(interior)))
    t = 2 * np.pi * rng.random(len(interior))
    interior = interior + np.stack([r * np.cos(t), r * np.sin(t)], axis=1)
    nb = int(np.round(side / s))
    e = np.linspace(0.0, side, nb + 1)
    bnd = np.concatenate([
        np.stack([e, np.zeros_like(e)], 1),                 # south
        np.stack([e[1:], np.full(nb, side)], 1),            # north
        np.stack([np.zeros(nb - 1), e[1:-1]], 1),           # west
        np.stack([np.full(nb - 1, side), e[1:-1]], 1),      # east
        np.array([[0.0, side]]),
    ])
    xy = np.concatenate([bnd, interior])
    tri = Delaunay(xy)
    cells = tri.simplices.astype(np.int32)
    used = np.zeros(len(xy), bool)
    used[cells] = True
    if not used.all():
        raise RuntimeError("Delaunay dropped %d vertices" % (~used).sum())
    # orient counter-clockwise
    p = xy[cells]
    area2 = (p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1]) - \
            (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1])
    flip = area2 < 0
    cells[flip] = cells[flip][:, [0, 2, 1]]
    coords = np.zeros((len(xy), 3))
    coords[:, :2] = xy
    onb = (np.isclose(xy[:, 0], 0.0) | np.isclose(xy[:, 0], side) |
           np.isclose(xy[:, 1], 0.0) | np.isclose(xy[:, 1], side))
    return coords, cells, onb


def icosphere(level, radius=EARTH_RADIUS):
    """Icosahedron refined `level` times; returns (coords, cells)."""
    phi = (1.0 + np.sqrt(5.0)) / 2.0
    v = np.array([[-1, phi, 0], [1, phi, 0], [-1, -phi, 0], [1, -phi, 0],
                  [0, -1, phi], [0, 1, phi], [0, -1, -phi], [0, 1, -phi],
                  [phi, 0, -1], [phi, 0, 1], [-phi, 0, -1], [-phi, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1)[:, None]
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
                  [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
                  [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                  [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    for _ in range(level):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * (len(v) + 1) + e[:, 1]
        uk, first, inv = np.unique(key, return_index=True, return_inverse=True)
        ue = e[first]
        mid = v[ue[:, 0]] + v[ue[:, 1]]
        mid /= np.linalg.norm(mid, axis=1)[:, None]
        base = len(v)
        v = np.concatenate([v, mid])
        nf = len(f)
        m01 = base + inv[:nf]
        m12 = base + inv[nf:2 * nf]
        m20 = base + inv[2 * nf:]
        f = np.concatenate([
            np.stack([f[:, 0], m01, m20], 1),
            np.stack([f[:, 1], m12, m01], 1),
            np.stack([f[:, 2], m20, m12], 1),
            np.stack([m01, m12, m20], 1)])
    return v * radius, f.astype(np.int32)


# ----------------------------------------------------------------------------
# fields
# ----------------------------------------------------------------------------
def fractal_field(xy, extent, seed, beta=2.0, ngrid=512):
    """k^-beta power spectrum noise on an ngrid^2 periodic grid, bilinear at xy."""
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(ngrid)[:, None]
    ky = np.fft.rfftfreq(ngrid)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    amp = k ** (-beta / 2.0)
    amp[0, 0] = 0.0
    spec = amp * (rng.standard_normal(amp.shape) + 1j * rng.standard_normal(amp.shape))
    grid = np.fft.irfft2(spec, s=(ngrid, ngrid))
    u = np.clip(xy[:, 0] / extent * (ngrid - 1), 0, ngrid - 1.000001)
    w = np.clip(xy[:, 1] / extent * (ngrid - 1), 0, ngrid - 1.000001)
    i0 = np.floor(u).astype(int)
    j0 = np.floor(w).astype(int)
    fu = u - i0
    fw = w - j0
    g = grid
    return ((1 - fu) * (1 - fw) * g[i0, j0] + fu * (1 - fw) * g[i0 + 1, j0] +
            (1 - fu) * fw * g[i0, j0 + 1] + fu * fw * g[i0 + 1, j0 + 1])


def _legendre_rows(lmax, sinlat, coslat):
    """Yield (m, P[l=m..lmax, nlat]) fully normalised associated Legendre."""
    pmm = np.ones_like(sinlat)
    for m in range(lmax + 1):
        if m > 0:
            pmm = pmm * coslat * np.sqrt((2.0 * m + 1.0) / (2.0 * m)) * (np.sqrt(2.0) if m == 1 else 1.0)
        rows = np.empty((lmax - m + 1, len(sinlat)))
        rows[0] = pmm
        if m < lmax:
            rows[1] = np.sqrt(2.0 * m + 3.0) * sinlat * pmm
        for l in range(m + 2, lmax + 1):
            a = np.sqrt((4.0 * l * l - 1.0) / (l * l - m * m))
            b = np.sqrt(((l - 1.0) ** 2 - m * m) / (4.0 * (l - 1.0) ** 2 - 1.0))
            rows[l - m] = a * (sinlat * rows[l - m - 1] - b * rows[l - m - 2])
        yield m, rows


def sh_field(coords, lmax, seed, beta=2.0, nlat=None):
    """Random real SH field (degrees 1..lmax, power ~ l^-beta) sampled at coords."""
    rng = np.random.default_rng(seed)
    nlat = nlat or max(2 * lmax + 2, 64)
    nlon = 2 * nlat
    lat = np.linspace(-np.pi / 2, np.pi / 2, nlat)
    sinlat, coslat = np.sin(lat), np.cos(lat)
    spec = np.zeros((nlat, nlon // 2 + 1), dtype=np.complex128)
    ls = np.arange(lmax + 1, dtype=np.float64)
    sig = np.zeros(lmax + 1)
    sig[1:] = np.sqrt(ls[1:] ** (-beta) / (2 * ls[1:] + 1))
    for m, rows in _legendre_rows(lmax, sinlat, coslat):
        a = rng.standard_normal(lmax - m + 1) * sig[m:]
        b = rng.standard_normal(lmax - m + 1) * sig[m:] if m > 0 else np.zeros(lmax - m + 1)
        fm_c = a @ rows
        fm_s = b @ rows
        spec[:, m] = (fm_c - 1j * fm_s) * (nlon if m > 0 else nlon) / (2.0 if m > 0 else 1.0)
    grid = np.fft.irfft(spec, n=nlon, axis=1)
    r = np.linalg.norm(coords, axis=1)
    la = np.arcsin(np.clip(coords[:, 2] / r, -1, 1))
    lo = np.mod(np.arctan2(coords[:, 1], coords[:, 0]), 2 * np.pi)
    u = (la + np.pi / 2) / np.pi * (nlat - 1)
    i0 = np.clip(np.floor(u).astype(int), 0, nlat - 2)
    fu = u - i0
    w = lo / (2 * np.pi) * nlon
    j0 = np.floor(w).astype(int) % nlon
    j1 = (j0 + 1) % nlon
    fw = w - np.floor(w)
    g = grid
    return ((1 - fu) * (1 - fw) * g[i0, j0] + fu * (1 - fw) * g[i0 + 1, j0] +
            (1 - fu) * fw * g[i0, j1] + fu * fw * g[i0 + 1, j1])


def rescale(f, lo, hi):
    f = np.asarray(f, dtype=np.float64)
    return lo + (f - f.min()) * (hi - lo) / (f.max() - f.min())


def belt_uplift(coords, seed, nbelt=3, halfwidth=500.0e3, amp=2.0e-3):
    """Sum of Gaussian belts around random great circles, clipped to +-amp (m/yr)."""
    rng = np.random.default_rng(seed)
    r = np.linalg.norm(coords, axis=1)
    u = coords / r[:, None]
    out = np.zeros(len(coords))
    for _ in range(nbelt):
        p = rng.standard_normal(3)
        p /= np.linalg.norm(p)
        a = rng.uniform(-amp, amp)
        d = np.abs(np.arcsin(np.clip(u @ p, -1, 1))) * r
        out += a * np.exp(-(d / halfwidth) ** 2)
    return np.clip(out, -amp, amp)


# ----------------------------------------------------------------------------
# workload recipes
# ----------------------------------------------------------------------------
def planar_config(n=20000, side=100.0e3, seed=20261204, zmax=50.0):
    """20k-vertex planar landscape: U = 1 mm/yr, P = 1 m/yr, K = 2e-6, flowdir 3."""
    coords, cells, onb = planar_hex_mesh(n, side, seed)
    z = rescale(fractal_field(coords[:, :2], side, seed + 1), 0.0, zmax)
    z[onb] = 0.0
    up = np.full(len(z), 1.0e-3)
    up[onb] = 0.0
    params = dict(dt=1000.0, tStart=0.0, tEnd=200 * 1000.0, flowDir=3, K=2.0e-6, d=0.0, m=0.5,
                  Cda=0.1, Cdm=0.1, sealevel=-100.0, oFill=-6000.0, bc="ffff")
    return coords, cells, z, np.ones(len(z)), up, params


def morton_order(coords):
    """Vertex permutation along a 3-D Morton (Z-order) curve of the positions,
    21 bits per axis over the bounding box: consecutive ids become spatial
    neighbours, so the neighbour gathers of every kernel hit the same cache
    lines."""
    lo = coords.min(axis=0)
    span = np.maximum(coords.max(axis=0) - lo, 1e-300)
    q = np.clip(((coords - lo) / span * ((1 << 21) - 1)).astype(np.uint64), 0, (1 << 21) - 1)

    def spread(x):
        x = x & np.uint64(0x1fffff)
        x = (x | (x << np.uint64(32))) & np.uint64(0x1f00000000ffff)
        x = (x | (x << np.uint64(16))) & np.uint64(0x1f0000ff0000ff)
        x = (x | (x << np.uint64(8))) & np.uint64(0x100f00f00f00f00f)
        x = (x | (x << np.uint64(4))) & np.uint64(0x10c30c30c30c30c3)
        x = (x | (x << np.uint64(2))) & np.uint64(0x1249249249249249)
        return x

    key = spread(q[:, 0]) | (spread(q[:, 1]) << np.uint64(1)) | (spread(q[:, 2]) << np.uint64(2))
    return np.argsort(key, kind="stable")


def renumber(coords, cells, order):
    """Mesh with vertex i of the result = vertex order[i] of the input; cells
    sorted by their smallest new vertex id."""
    inv = np.empty(len(order), np.int64)
    inv[order] = np.arange(len(order))
    c2 = inv[cells]
    c2 = c2[np.argsort(c2.min(axis=1), kind="stable")]
    return coords[order], c2.astype(cells.dtype)


def sphere_config(level=9, seed=20261205, lmax=256, zlo=-4000.0, zhi=3000.0, steps=50, dt=1.0e4,
                  K=5.0e-7, kd=0.05, ordered=True):
    """Icosahedral sphere: SH(l<=lmax, l^-2) relief, lognormal rain, three uplift
    belts.  With `ordered` the vertices are numbered along a Morton curve
    (the same landscape; only the numbering differs)."""
    coords, cells = icosphere(level)
    if ordered:
        coords, cells = renumber(coords, cells, morton_order(coords))
    z = rescale(sh_field(coords, lmax, seed + 1), zlo, zhi)
    g = sh_field(coords, 32, seed + 2)
    g = (g - g.mean()) / g.std()
    rain = np.exp(0.5 * g)
    up = belt_uplift(coords, seed + 3)
    params = dict(dt=dt, tStart=0.0, tEnd=steps * dt, flowDir=3, K=K, d=0.0, m=0.5,
                  Cda=kd, Cdm=kd, sealevel=0.0, oFill=-6000.0, bc="oooo")
    return coords, cells, z, rain, up, params


def gp_field(xy, extent, seed, ell, ngrid=512):
    """Seeded stationary Gaussian field with squared-exponential covariance
    exp(-r^2 / (2 ell^2)) at the points xy of [0, extent]^2: white noise on a
    periodic ngrid^2 grid over twice the extent (so the period exceeds the
    domain plus the correlation length), filtered by the square root of the
    covariance's spectral density exp(-2 pi^2 ell^2 |f|^2), bilinear at xy;
    unit variance."""
    rng = np.random.default_rng(seed)
    span = 2.0 * extent
    f = np.fft.fftfreq(ngrid, d=span / ngrid)
    fx = f[:, None]
    fy = np.fft.rfftfreq(ngrid, d=span / ngrid)[None, :]
    amp = np.exp(-np.pi ** 2 * ell ** 2 * (fx * fx + fy * fy))
    noise = np.fft.rfft2(rng.standard_normal((ngrid, ngrid)))
    grid = np.fft.irfft2(noise * amp, s=(ngrid, ngrid))
    grid = (grid - grid.mean()) / grid.std()
    u = np.clip(xy[:, 0] / span * ngrid, 0, ngrid - 1.000001)
    w = np.clip(xy[:, 1] / span * ngrid, 0, ngrid - 1.000001)
    i0 = np.floor(u).astype(int)
    j0 = np.floor(w).astype(int)
    fu = u - i0
    fw = w - j0
    g = grid
    return ((1 - fu) * (1 - fw) * g[i0, j0] + fu * (1 - fw) * g[i0 + 1, j0] +
            (1 - fu) * fw * g[i0, j0 + 1] + fu * fw * g[i0 + 1, j0 + 1])


def adjoint_config(n=160000, side=200.0e3, seed=20261207):
    """Inversion for erodibility: a jittered-hex planar mesh of ~n vertices over
    side x side, fractal initial relief 0-100 m with fixed boundary vertices at
    0, uplift 0.5 mm/yr (none on the boundary), rain 1 m/yr, dt 1000 yr, and
    the hidden 'true' erodibility: ln K a Gaussian field (correlation length
    20 km) scaled to -14..-11.  Returns coords, cells, z, rain, uplift,
    params (K = the true field), the boundary mask and the uniform start
    K0 = exp(-12.5)."""
    coords, cells, onb = planar_hex_mesh(n, side, seed)
    z = rescale(fractal_field(coords[:, :2], side, seed + 1), 0.0, 100.0)
    z[onb] = 0.0
    lnk = rescale(gp_field(coords[:, :2], side, seed + 2, 20.0e3), -14.0, -11.0)
    up = np.full(len(z), 5.0e-4)
    up[onb] = 0.0
    params = dict(dt=1000.0, tStart=0.0, tEnd=100 * 1000.0, flowDir=3, K=np.exp(lnk), d=0.0, m=0.5,
                  Cda=0.1, Cdm=0.1, sealevel=-100.0, oFill=-6000.0, bc="ffff")
    return coords, cells, z, np.ones(len(z)), up, params, onb, float(np.exp(-12.5))


def ensemble_member(n, seed, spacing=250.0):
    """One ensemble landscape: ~n vertices at `spacing`, own K, rain and relief."""
    rng = np.random.default_rng(seed)
    side = spacing * np.sqrt(n * np.sqrt(3.0) / 2.0)
    coords, cells, onb = planar_hex_mesh(n, side, seed)
    z = rescale(fractal_field(coords[:, :2], side, seed + 1), 0.0, 100.0)
    z[onb] = 0.0
    g = fractal_field(coords[:, :2], side, seed + 2, beta=4.0)
    g = (g - g.mean()) / g.std()
    rain = np.exp(0.7 * g)
    K = float(np.exp(rng.uniform(np.log(1e-7), np.log(1e-5))))
    params = dict(dt=500.0, tStart=0.0, tEnd=100 * 500.0, flowDir=3, K=K, d=0.0, m=0.5,
                  Cda=0.1, Cdm=0.1, sealevel=-100.0, oFill=-6000.0, bc="ffff")
    return coords, cells, z, rain, np.zeros(len(z)), params


def ensemble_sizes(count=256, lo=1.0e4, hi=5.0e5, seed=20261206):
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(int)
