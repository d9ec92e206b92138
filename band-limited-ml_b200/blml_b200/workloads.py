"""Seeded synthetic inputs with the shapes of the binned path's workloads (NumPy on the host, so the GPU path and
any CPU checker see identical arrays). There is no public dataset on this path; every workload is generated.

  lattice_1d_mixture   1,024-bin histogram of n = 1e5 draws of a 3-component Gaussian mixture (means .3/.5/.7, sd .05,
                       weights .3/.4/.3), clipped to [0, 1): the 1-D sinc fit.
  two_disk_field       counts ~ Poisson(N p) on an (M1, M2) torus, p = 0.95 |h|^2 / sum |h|^2 + 0.05 / (M1 M2), h the
                       inverse DFT of two displaced disks in the band with a random relative phase: the pball fits.
  cutoff_sweep         64 such fits of uneven size and cut-off with an 80/20 binomial held-out split.
  warm_start_set       128 x 128 fits of two-disk (pball kernel) or two-slit (slits x sinc kernel) fields for the
                       learned warm start.
  points_5d_mixture    n = 2e5 points of an 8-component 5-D Gaussian mixture in the unit cube for the pair path.
"""
import numpy as np

SIDES = (64, 96, 128, 192, 256, 384)


def lattice_1d_mixture(seed=0, n=100_000, m=1024):
    rng = np.random.default_rng(seed)
    comp = rng.choice(3, n, p=[0.3, 0.4, 0.3])
    x = np.array([0.3, 0.5, 0.7])[comp] + 0.05 * rng.standard_normal(n)
    x = np.clip(x, 0.0, np.nextafter(1.0, 0.0))
    return np.bincount(np.floor(x * m).astype(np.int64), minlength=m).astype(np.float64)


def two_disk_field(shape=(256, 256), fc=0.33, N=1e6, seed=0, diameter=None, shift=None, bg=0.05):
    """Counts on an (M1, M2) torus from a field whose spectrum is two disks of diameter `diameter` (cycles/bin,
    default fc / 2) displaced by +-shift along axis 0 (default fc / 4), so both lie inside the pball band of
    cut-off fc, with a uniformly random relative phase."""
    rng = np.random.default_rng(seed)
    M1, M2 = shape
    diameter = fc / 2 if diameter is None else diameter
    shift = fc / 4 if shift is None else shift
    k1 = np.fft.fftfreq(M1)[:, None]; k2 = np.fft.fftfreq(M2)[None, :]
    r = diameter / 2
    A = ((k1 - shift) ** 2 + k2 ** 2 <= r * r).astype(complex)
    A = A + np.exp(2j * np.pi * rng.uniform()) * ((k1 + shift) ** 2 + k2 ** 2 <= r * r)
    h = np.fft.ifft2(A)
    p = (1 - bg) * np.abs(h) ** 2 / np.sum(np.abs(h) ** 2) + bg / (M1 * M2)
    return rng.poisson(N * p).astype(np.float64)


def two_slit_field(shape=(128, 128), fc=0.25, N=1e5, seed=0, bg=0.05):
    """Counts on an (M1, M2) lattice from a field whose spectrum is two slits at +-3 fc / 8 along axis 0 (width
    fc / 8) of height fc / 2 along axis 1 (rounded to DFT bins, at least one bin), with a uniformly random relative
    phase: inside the band of slits_modes(shape, fc)."""
    rng = np.random.default_rng(seed)
    M1, M2 = shape
    # in DFT bins, at least one bin wide (a slit narrower than the grid would be empty on small lattices)
    i1 = np.fft.fftfreq(M1, 1.0 / M1)[:, None]; i2 = np.fft.fftfreq(M2, 1.0 / M2)[None, :]
    d = max(1, int(round(3 * fc / 8 * M1))); a = int(round(fc / 16 * M1)); b = int(round(fc / 4 * M2))
    A = ((np.abs(i1 - d) <= a) & (np.abs(i2) <= b)).astype(complex)
    A = A + np.exp(2j * np.pi * rng.uniform()) * ((np.abs(i1 + d) <= a) & (np.abs(i2) <= b))
    h = np.fft.ifft2(A)
    p = (1 - bg) * np.abs(h) ** 2 / np.sum(np.abs(h) ** 2) + bg / (M1 * M2)
    return rng.poisson(N * p).astype(np.float64)


def slits_modes(shape, fc, fill=0.5):
    """A product mode: two slits (band fc (1 - fill) / 2 <= |nu| <= fc / 2) on axis 0, sinc of cut-off fc on axis 1."""
    return [{0: dict(kind='slits', fc=float(fc), fill=float(fill)), 1: dict(kind='sinc', fc=float(fc))}]


def warm_start_set(n, seed=0, shape=(128, 128)):
    """Fits of the warm-start workload: fit i draws, with default_rng(seed + i), a pupil (two disks under a pball
    kernel or two slits under a slits x sinc kernel), fc ~ U(0.1, 0.4) and N = 10^U(4, 6)."""
    out = []
    for i in range(n):
        rng = np.random.default_rng(seed + i)
        kind = 'pball' if rng.uniform() < 0.5 else 'slits'
        fc = float(rng.uniform(0.1, 0.4)); N = float(10 ** rng.uniform(4, 6))
        if kind == 'pball':
            counts = two_disk_field(shape, fc=fc, N=N, seed=seed + 7919 * (i + 1))
            modes = pball_modes(shape, fc)
        else:
            counts = two_slit_field(shape, fc=fc, N=N, seed=seed + 7919 * (i + 1))
            modes = slits_modes(shape, fc)
        out.append(dict(kind=kind, fc=fc, N=N, counts=counts, modes=modes))
    return out


def pball_modes(shape, fc, bg_fc=None):
    """The signal pball mode over both columns with the lattice as its period, plus an optional background pball."""
    per = [float(shape[0]), float(shape[1])]
    modes = [{(0, 1): dict(kind='pball', fc=float(fc), period=per)}]
    if bg_fc is not None:
        modes.append({(0, 1): dict(kind='pball', fc=float(bg_fc), period=per)})
    return modes


def cutoff_sweep(seed=0, n_fits=64):
    """Fit i: sides from SIDES, fc from geomspace(0.05, 0.45, 16), N = 10^U(4, 6), drawn with default_rng(seed + i);
    train = Binomial(counts, 0.8), held-out = counts - train."""
    grid = np.geomspace(0.05, 0.45, 16)
    fits = []
    for i in range(n_fits):
        rng = np.random.default_rng(seed + i)
        M1, M2 = int(rng.choice(SIDES)), int(rng.choice(SIDES))
        fc = float(rng.choice(grid)); N = float(10 ** rng.uniform(4, 6))
        counts = two_disk_field((M1, M2), fc=fc, N=N, seed=seed + 1000 + i)
        train = rng.binomial(counts.astype(np.int64), 0.8).astype(np.float64)
        fits.append(dict(shape=(M1, M2), fc=fc, N=N, counts=counts, train=train, val=counts - train))
    return fits


def points_5d_mixture(seed=0, n=200_000, d=5, comps=8):
    rng = np.random.default_rng(seed)
    means = rng.uniform(0.2, 0.8, (comps, d)); sds = rng.uniform(0.03, 0.1, (comps, d))
    wts = rng.dirichlet(np.ones(comps))
    c = rng.choice(comps, n, p=wts)
    X = means[c] + sds[c] * rng.standard_normal((n, d))
    return np.clip(X, 0.0, np.nextafter(1.0, 0.0))


def two_blob_points(n=200_000, seed=0):
    """n points in the unit square from two Gaussian blobs (60% at (0.35, 0.4), sd 0.08; 40% at (0.7, 0.75), sd 0.05);
    the second column wrapped into [0, 1) (a periodic column of period 1)."""
    rng = np.random.default_rng(seed)
    comp = rng.uniform(size=n) < 0.6
    X = np.where(comp[:, None], rng.normal([0.35, 0.4], 0.08, (n, 2)), rng.normal([0.7, 0.75], 0.05, (n, 2)))
    X[:, 1] = np.mod(X[:, 1], 1.0)
    return X
