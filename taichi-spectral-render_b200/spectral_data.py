"""Spectral data for the host side: loaders with the reference's interface
(data.py:6-182) and analytic generators for the synthetic workloads.

Loaders (same constructor arguments and attributes as the reference's classes):
  RefractiveIndex  refractiveindex.info "tabulated nk" YAML -> .n, .k per band
  ColourSystem     CMF table + primaries/white -> .cmf [B][3], .T (XYZ->RGB),
                   .normalization_factor
  SpecularVec      two-column spectrum -> .vec per band (times scale)
  EEMMatrix        excitation/emission grid -> .matrix [B][B] with the Stokes
                   mask, ids handed out from a class counter starting at 1

Generators:
  cie1931_fit      multi-lobe piecewise-Gaussian fit of the CIE 1931 2-degree
                   observer (Wyman, Sloan, Shirley, "Simple Analytic
                   Approximations to the CIE XYZ Color Matching Functions",
                   JCGT 2(2), 2013)
  planck           blackbody spectral radiance shape
  cauchy_n         n(lambda) = A + B / lambda^2 (lambda in micrometres)
  logistic         sigmoid reflectance spectra
  reflectance_to_k extinction coefficient that makes the reference's diffuse
                   albedo sigma_s / (sigma_s + 4 pi k / lambda) equal a
                   reflectance when sigma_s = 1
  gaussian_stokes_eem  excitation-emission matrix with a Gaussian Stokes shift
"""
import numpy as np


# --------------------------------------------------------------------------- loaders
def _targets(wavelength_min, wavelength_max, spectral_bands):
    return np.linspace(wavelength_min, wavelength_max, spectral_bands)


class RefractiveIndex:
    """n and k of a refractiveindex.info YAML file at the band centres."""

    def __init__(self, file_path, wavelength_min, wavelength_max, spectral_bands):
        import yaml
        self.file_path = file_path
        self.target_wavelengths_nm = _targets(wavelength_min, wavelength_max, spectral_bands)
        with open(file_path) as fh:
            doc = yaml.safe_load(fh)
        table = None
        for entry in doc.get("DATA", []):
            if entry.get("type") == "tabulated nk":
                table = entry.get("data")
                break
        if not table:
            raise ValueError(f"{file_path}: no 'tabulated nk' block")
        rows = []
        for line in table.strip().split("\n"):
            parts = line.split()
            if len(parts) != 3:
                continue
            try:
                rows.append([float(p) for p in parts])
            except ValueError:
                continue
        arr = np.asarray(rows, dtype=np.float64)
        wl_nm = arr[:, 0] * 1000.0
        order = np.argsort(wl_nm)
        wl_nm, n, k = wl_nm[order], arr[order, 1], arr[order, 2]
        self.n = np.interp(self.target_wavelengths_nm, wl_nm, n).tolist()
        self.k = np.interp(self.target_wavelengths_nm, wl_nm, k).tolist()


def _xyz_from_xy(xy):
    return np.array((xy[0], xy[1], 1.0 - xy[0] - xy[1]))


def xyz_to_rgb_matrix(red, green, blue, white):
    """XYZ -> linear RGB for the given chromaticities (white-point scaled)."""
    M = np.vstack((_xyz_from_xy(red), _xyz_from_xy(green), _xyz_from_xy(blue))).T
    MI = np.linalg.inv(M)
    wscale = MI.dot(_xyz_from_xy(white))
    return MI / wscale[:, np.newaxis]


def srgb_xyz_to_rgb():
    """The reference's display primaries (main.py:55-64)."""
    return xyz_to_rgb_matrix([0.64, 0.33], [0.30, 0.60], [0.15, 0.06], [0.33242, 0.34743])


class ColourSystem:
    """Colour-matching functions resampled to the bands plus the XYZ->RGB matrix."""

    def __init__(self, file_path, red, green, blue, white, wavelength_min, wavelength_max, spectral_bands):
        self.red, self.green, self.blue, self.white = (_xyz_from_xy(red), _xyz_from_xy(green), _xyz_from_xy(blue),
                                                       _xyz_from_xy(white))
        self.M = np.vstack((self.red, self.green, self.blue)).T
        self.MI = np.linalg.inv(self.M)
        self.wscale = self.MI.dot(self.white)
        self.T = self.MI / self.wscale[:, np.newaxis]
        self.cmf_raw = np.loadtxt(file_path, comments="#")
        self.target_wavelengths = _targets(wavelength_min, wavelength_max, spectral_bands)
        src = self.cmf_raw[:, 0]
        self.cmf = np.stack([np.interp(self.target_wavelengths, src, self.cmf_raw[:, 1 + c]) for c in range(3)],
                            axis=1)
        self.wavelength_step = (wavelength_max - wavelength_min) / (spectral_bands - 1)
        self.normalization_factor = np.sum(self.cmf[:, 1]) * self.wavelength_step


class SpecularVec:
    """A two-column spectrum resampled to the bands and scaled."""

    def __init__(self, file_path, scale, wavelength_min, wavelength_max, spectral_bands):
        self.raw = np.loadtxt(file_path, comments="#")
        self.target_wavelengths = _targets(wavelength_min, wavelength_max, spectral_bands)
        self.vec = (np.interp(self.target_wavelengths, self.raw[:, 0], self.raw[:, 1]) * scale).tolist()


class EEMMatrix:
    """Excitation-emission matrix [excitation][emission] at the band centres.

    From a file (first row: emission axis, first column: excitation axis) the
    grid is resampled with a bicubic tensor spline, emission <= excitation is
    zeroed (Stokes shift) and negatives are clipped.  ``id`` numbers matrices
    in creation order starting at 1 (0 means "no fluorescence").
    """
    _next_eem_id = 1

    def __init__(self, wavelength_min, wavelength_max, spectral_bands, file_path=None, matrix=None):
        self.target_wavelengths = _targets(wavelength_min, wavelength_max, spectral_bands)
        if file_path:
            from scipy.interpolate import RectBivariateSpline
            raw = np.loadtxt(file_path, comments="#")
            spline = RectBivariateSpline(raw[1:, 0], raw[0, 1:], raw[1:, 1:])
            m = spline(self.target_wavelengths, self.target_wavelengths)
            lam = self.target_wavelengths
            m[lam[None, :] <= lam[:, None]] = 0.0
            self.matrix = np.maximum(0, m)
        elif matrix is not None:
            self.matrix = np.asarray(matrix, dtype=np.float64)
        else:
            raise ValueError("EEMMatrix needs file_path or matrix")
        self.id = EEMMatrix._next_eem_id
        EEMMatrix._next_eem_id += 1


# --------------------------------------------------------------------------- generators
def _pw_gauss(x, mu, s1, s2):
    s = np.where(x < mu, s1, s2)
    return np.exp(-0.5 * ((x - mu) / s) ** 2)


def cie1931_fit(wavelengths_nm):
    """[B][3] x-bar, y-bar, z-bar from the multi-lobe fit of Wyman et al. 2013."""
    x = np.asarray(wavelengths_nm, dtype=np.float64)
    xb = 1.056 * _pw_gauss(x, 599.8, 37.9, 31.0) + 0.362 * _pw_gauss(x, 442.0, 16.0, 26.7) \
        - 0.065 * _pw_gauss(x, 501.1, 20.4, 26.2)
    yb = 0.821 * _pw_gauss(x, 568.8, 46.9, 40.5) + 0.286 * _pw_gauss(x, 530.9, 16.3, 31.1)
    zb = 1.217 * _pw_gauss(x, 437.0, 11.8, 36.0) + 0.681 * _pw_gauss(x, 459.0, 26.0, 13.8)
    return np.stack([xb, yb, zb], axis=1)


def planck(wavelengths_nm, temperature_k):
    """Blackbody spectral radiance (arbitrary units, unnormalised)."""
    h, c, kb = 6.62607015e-34, 2.99792458e8, 1.380649e-23
    lam = np.asarray(wavelengths_nm, dtype=np.float64) * 1e-9
    return (2 * h * c * c / lam ** 5) / np.expm1(h * c / (lam * kb * temperature_k))


def cauchy_n(wavelengths_nm, a=1.5, b=0.0042):
    lam_um = np.asarray(wavelengths_nm, dtype=np.float64) * 1e-3
    return a + b / lam_um ** 2


def logistic(wavelengths_nm, centre, slope):
    return 1.0 / (1.0 + np.exp(-slope * (np.asarray(wavelengths_nm, dtype=np.float64) - centre)))


def reflectance_to_k(rho, wavelengths_nm, lo=0.01, hi=0.99):
    """k with 4 pi k / lambda = 1/rho - 1 (so sigma_s = 1 gives albedo rho)."""
    r = np.clip(np.asarray(rho, dtype=np.float64), lo, hi)
    lam_m = np.asarray(wavelengths_nm, dtype=np.float64) * 1e-9
    return lam_m * (1.0 / r - 1.0) / (4.0 * np.pi)


def absorption_to_k(sigma_a, wavelengths_nm):
    """k for an absorption coefficient sigma_a [1/m]: sigma_a = 4 pi k / lambda."""
    return np.asarray(sigma_a, dtype=np.float64) * np.asarray(wavelengths_nm, dtype=np.float64) * 1e-9 / (4 * np.pi)


def gaussian_stokes_eem(wavelengths_nm, shift_nm=40.0, width_nm=15.0, quantum_yield=0.6):
    """[excitation][emission] matrix: a Gaussian in (emission - excitation - shift),
    zero where emission < excitation, each non-empty row scaled so that its
    maximum (the reference's acceptance probability) equals quantum_yield."""
    lam = np.asarray(wavelengths_nm, dtype=np.float64)
    d = lam[None, :] - lam[:, None]
    m = np.exp(-0.5 * ((d - shift_nm) / width_nm) ** 2)
    m[d < 0] = 0.0
    rmax = m.max(axis=1, keepdims=True)
    with np.errstate(invalid="ignore", divide="ignore"):
        m = np.where(rmax > 0, m / rmax * quantum_yield, 0.0)
    return m
