"""LISA orbit tables for the fast frequency-domain response.

The reference response kernel reads spacecraft positions and link unit vectors from an
external lisatools ``Orbits`` object (``Response.cu:86-133``; tables pushed through
``AddOrbits::add_orbit_information(dt, N, n_arr, L_arr, x_arr, links, sc_r, sc_e,
armlength)``, ``lisaresponse.pyx:12``, ``fastfdresponse.py:104-105``).  lisatools and its
orbit file are not part of this project, so :class:`EqualArmlengthOrbits` builds the
same kind of table from the analytic first-order-in-eccentricity LISA orbit
(Rubbo, Cornish & Poujade 2004, eq. 57):

    x_k = a cos(alpha) + a e (sin(alpha) cos(alpha) sin(b_k) - (1 + sin^2 alpha) cos(b_k))
    y_k = a sin(alpha) + a e (sin(alpha) cos(alpha) cos(b_k) - (1 + cos^2 alpha) sin(b_k))
    z_k = -sqrt(3) a e cos(alpha - b_k)

with alpha = Omega0 t, b_k = 2 pi (k - 1) / 3, a = 1 AU and e = L / (2 sqrt(3) a).
Link ``ij`` (receiver i, emitter j) has unit vector n_ij = (x_i - x_j) / |x_i - x_j|.

Layout (shared with the CUDA lookup in ``bbhx_b200/csrc/bbhx_orbits.cuh``):
``x_arr[N, 3, 3]``, ``n_arr[N, 6, 3]``, ``L_arr[N, 6]``, sample k at t = k dt, linear
interpolation inside [0, (N-1) dt), zero vector outside.
"""
import numpy as np

from .utils.constants import AU_SI, L_SI, Omega0, YRSID_SI


class _HostBackendName:
    """Minimal ``backend`` attribute (``fastfdresponse.py:175`` compares backend names)."""

    name = "bbhx_b200_cuda"


class Orbits:
    """Base class of orbit tables consumed by :class:`LISATDIResponse`."""

    LINKS = [12, 23, 31, 13, 32, 21]
    SC = [1, 2, 3]

    def __init__(self, t_base, x_arr, n_arr, L_arr, armlength):
        self.t_base = np.asarray(t_base, dtype=np.float64)
        self.dt = float(self.t_base[1] - self.t_base[0])
        self.N = int(len(self.t_base))
        self.x_arr = np.ascontiguousarray(x_arr, dtype=np.float64).reshape(self.N, 3, 3)
        self.n_arr = np.ascontiguousarray(n_arr, dtype=np.float64).reshape(self.N, 6, 3)
        self.L_arr = np.ascontiguousarray(L_arr, dtype=np.float64).reshape(self.N, 6)
        self.armlength = float(armlength)
        self.links = np.asarray(self.LINKS, dtype=np.int32)
        self.sc_r = np.asarray([int(str(li)[0]) for li in self.LINKS], dtype=np.int32)
        self.sc_e = np.asarray([int(str(li)[1]) for li in self.LINKS], dtype=np.int32)
        self.backend = _HostBackendName()
        self.configured = False

    def configure(self, linear_interp_setup=True, **kwargs):
        """Kept for call compatibility (``fastfdresponse.py:174``); tables are ready."""
        self.configured = True
        return self

    @property
    def pycppdetector_args(self):
        """The nine ``add_orbit_information`` arguments, in the reference's order."""
        return (
            self.dt,
            self.N,
            self.n_arr.ravel(),
            self.L_arr.ravel(),
            self.x_arr.ravel(),
            self.links,
            self.sc_r,
            self.sc_e,
            self.armlength,
        )

    # host-side evaluation with the same lookup rule as the device code (used by tests)
    def _lerp(self, tab, t):
        t = np.asarray(t, dtype=np.float64)
        w = np.floor(t / self.dt)
        ok = (w >= 0) & (w < self.N - 1)
        wi = np.where(ok, w, 0).astype(np.int64)
        lo = tab[wi]
        hi = tab[wi + 1]
        tt = (t - wi * self.dt)[..., None]
        val = lo + (hi - lo) / self.dt * tt
        return np.where(ok[..., None], val, 0.0)

    def get_pos(self, t, sc):
        return self._lerp(self.x_arr[:, sc - 1, :], t)

    def get_normal_unit_vec(self, t, link):
        li = self.LINKS.index(link)
        return self._lerp(self.n_arr[:, li, :], t)


class EqualArmlengthOrbits(Orbits):
    """Analytic equal-armlength LISA orbit sampled every ``dt`` seconds.

    Args:
        dt: table spacing in seconds (default 1e4 s).
        t_max_years: table span in years starting at t = 0 (default 10).
        armlength: nominal armlength in m (default 2.5e9, the reference's ``L_SI``).
    """

    def __init__(self, dt=1.0e4, t_max_years=10.0, armlength=L_SI, force_backend=None):
        n = int(np.ceil(t_max_years * YRSID_SI / dt)) + 1
        t = np.arange(n, dtype=np.float64) * dt
        a = AU_SI
        e = armlength / (2.0 * np.sqrt(3.0) * a)
        alpha = Omega0 * t
        ca, sa = np.cos(alpha), np.sin(alpha)
        x = np.empty((n, 3, 3))
        for k in range(3):
            b = 2.0 * np.pi * k / 3.0
            cb, sb = np.cos(b), np.sin(b)
            x[:, k, 0] = a * ca + a * e * (sa * ca * sb - (1.0 + sa * sa) * cb)
            x[:, k, 1] = a * sa + a * e * (sa * ca * cb - (1.0 + ca * ca) * sb)
            x[:, k, 2] = -np.sqrt(3.0) * a * e * np.cos(alpha - b)
        n_arr = np.empty((n, 6, 3))
        L_arr = np.empty((n, 6))
        for li, link in enumerate(self.LINKS):
            r, s = int(str(link)[0]) - 1, int(str(link)[1]) - 1
            d = x[:, r, :] - x[:, s, :]
            ln = np.sqrt(np.sum(d * d, axis=1))
            n_arr[:, li, :] = d / ln[:, None]
            L_arr[:, li] = ln
        super().__init__(t, x, n_arr, L_arr, armlength)
