"""Uneven batches: many independent likelihood problems evaluated together.

A batch holds
  * direct groups — a ``Likelihood`` (its own data stream, hence its own observation span and
    data grid), binaries ``params`` [12, n], a sparse-grid ``length`` and a mode set;
  * heterodyned groups — a ``HeterodynedLikelihood`` (its own relative-binning grid of any
    length) and walkers [12, n].
``run()`` builds every group's inputs on the device -- sparse buffers and splines of the direct
groups, per-walker model records of the heterodyned ones -- then evaluates ALL groups of a
precision class in ONE persistent launch (``bbhx_uneven_like``): the heterodyned walkers and the
direct (data tile, binary) items form one work range.  Nothing in ``run()`` synchronises with
the host, so ``capture()`` records it once in a CUDA graph and ``replay()`` re-runs it
(parameters are updated in place with ``set_params``).  The launch shape of the persistent
kernel (data bins per work item, CTAs per SM) is chosen by ``Autotuner`` by timing the
candidates on the batch.

No reference counterpart: the reference evaluates one problem per call.
"""
import ctypes
import itertools

from . import _lib
from .utils.arrays import device, torch
from .utils.constants import YRSID_SI
from .likelihood import pack_lnl
from .waveformbuild import PRECISIONS


class DirectGroupC(ctypes.Structure):
    """Mirror of ``bbhx_direct_group`` (include/bbhx_b200.h)."""

    _fields_ = [("data_freqs", ctypes.c_void_p), ("data", ctypes.c_void_p),
                ("noise", ctypes.c_void_p), ("data_length", ctypes.c_int),
                ("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("c1", ctypes.c_void_p),
                ("c2", ctypes.c_void_p), ("c3", ctypes.c_void_p),
                ("t_start", ctypes.c_void_p), ("t_end", ctypes.c_void_p),
                ("num_modes", ctypes.c_int), ("length", ctypes.c_int),
                ("num_bin_all", ctypes.c_int), ("d_h", ctypes.c_void_p), ("h_h", ctypes.c_void_p),
                ("data32", ctypes.c_void_p), ("noise32", ctypes.c_void_p)]


class HdynGroupC(ctypes.Structure):
    """Mirror of ``bbhx_hdyn_group`` (include/bbhx_b200.h)."""

    _fields_ = [("orbits", ctypes.c_void_p), ("d_h", ctypes.c_void_p), ("h_h", ctypes.c_void_p),
                ("coeffs", ctypes.c_void_p), ("ells", ctypes.c_void_p), ("mms", ctypes.c_void_p),
                ("phi_ref", ctypes.c_void_p), ("inc", ctypes.c_void_p), ("lam", ctypes.c_void_p),
                ("beta", ctypes.c_void_p), ("psi", ctypes.c_void_p), ("t_ref", ctypes.c_void_p),
                ("t_init", ctypes.c_double), ("t_start", ctypes.c_void_p),
                ("t_end", ctypes.c_void_p), ("freqs", ctypes.c_void_p), ("h0", ctypes.c_void_p),
                ("consts", ctypes.c_void_p), ("TDItag", ctypes.c_int), ("rescaled", ctypes.c_int),
                ("tdi2", ctypes.c_int), ("num_modes", ctypes.c_int), ("length", ctypes.c_int),
                ("num_bin_all", ctypes.c_int)]


class HdynSourceC(ctypes.Structure):
    """Mirror of ``bbhx_hdyn_source`` (include/bbhx_b200.h)."""

    _fields_ = [("group", HdynGroupC), ("params", ctypes.c_void_p), ("qnm_table", ctypes.c_void_p),
                ("qnm_n", ctypes.c_int), ("dspin", ctypes.c_double),
                ("t_obs_start_L", ctypes.c_double), ("t_obs_end_L", ctypes.c_double),
                ("run_phenomd", ctypes.c_int), ("flags", ctypes.c_void_p)]


class DirectSourceC(ctypes.Structure):
    """Mirror of ``bbhx_direct_source`` (include/bbhx_b200.h)."""

    _P, _D, _I = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
    _fields_ = [("orbits", _P), ("params", _P), ("ells", _P), ("mms", _P), ("qnm_table", _P),
                ("qnm_n", _I), ("dspin", _D), ("mf_min", _D), ("mf_max", _D), ("t_init", _D),
                ("t_obs_start_L", _D), ("t_obs_end_L", _D), ("orbit_tmin", _D),
                ("orbit_tmax", _D), ("TDItag", _I), ("rescaled", _I), ("tdi2", _I),
                ("run_phenomd", _I), ("num_modes", _I), ("length", _I), ("num_bin_all", _I),
                ("x", _P), ("y", _P), ("c1", _P), ("c2", _P), ("c3", _P), ("t_start", _P),
                ("t_end", _P), ("flags", _P), ("data_freqs", _P), ("data", _P), ("noise", _P),
                ("data_length", _I), ("data32", _P), ("noise32", _P), ("d_h", _P), ("h_h", _P)]


class DirectGroup:
    def __init__(self, like, params, length=1024, modes=None, t_obs_start=0.0, t_obs_end=1.0):
        t = torch()
        self.like = like
        self.params = t.as_tensor(params, dtype=t.float64, device=device()).contiguous()
        self.length, self.modes = length, modes
        self.t_obs_start, self.t_obs_end = t_obs_start, t_obs_end
        self.flags = t.zeros(3, dtype=t.int32, device=device())

    @property
    def size(self):
        return self.params.shape[1]

    def source(self, precision="fp64"):
        """Descriptor of this group for bbhx_uneven_batch: its parameters and model settings,
        and the device buffers the batch's sparse build and likelihood write (allocated here;
        no host synchronisation)."""
        from .waveforms.ringdownphenomd import dspin

        t = torch()
        wave = self.like.waveform_gen
        ap, rg = wave.amp_phase_gen, wave.response_gen
        ells, mms = ap.mode_tensors(self.modes)
        B, M, L = self.size, int(ells.numel()), self.length
        n = B * M * L
        f64 = dict(dtype=t.float64, device=device())
        x, y = t.empty(n, **f64), t.empty(9 * n, **f64)
        c1, c2, c3 = t.empty(9 * n, **f64), t.empty(9 * n, **f64), t.empty(9 * n, **f64)
        ts, te = t.empty(B, **f64), t.empty(B, **f64)
        self.M, self.L = M, L
        self.d_h = t.empty(B, dtype=t.complex128, device=device())
        self.h_h = t.empty(B, dtype=t.complex128, device=device())
        self.packed = t.empty(3 * B, **f64)
        lk = self.like
        d32, n32 = lk.fp32_data() if precision == "mixed" else (None, None)
        tab = ap.qnm_table
        self._keep = (x, y, c1, c2, c3, ts, te, ells, mms, tab)
        p = lambda a: _lib.dptr(a).value if a is not None else None  # noqa: E731
        return DirectSourceC(
            orbits=rg.orbit_handle.ptr.value, params=p(self.params), ells=p(ells), mms=p(mms),
            qnm_table=p(tab), qnm_n=int(tab.shape[1]), dspin=float(dspin),
            mf_min=float(ap.mf_min), mf_max=float(ap.mf_max), t_init=float(ap.initial_t_val),
            t_obs_start_L=float(self.t_obs_start * YRSID_SI),
            t_obs_end_L=float(self.t_obs_end * YRSID_SI),
            orbit_tmin=float(rg.orbits.t_base.min()), orbit_tmax=float(rg.orbits.t_base.max()),
            TDItag=rg.TDItag_int, rescaled=int(rg.rescaled), tdi2=int(rg.tdi2),
            run_phenomd=int(ap.run_phenomd), num_modes=M, length=L, num_bin_all=B, x=p(x),
            y=p(y), c1=p(c1), c2=p(c2), c3=p(c3), t_start=p(ts), t_end=p(te),
            flags=p(self.flags), data_freqs=p(lk.data_freqs), data=p(lk.data_channels),
            noise=p(lk.noise_factors), data_length=int(lk.data_freqs.numel()), data32=p(d32),
            noise32=p(n32), d_h=p(self.d_h), h_h=p(self.h_h))

    def lnl(self):
        return pack_lnl(self.d_h, self.h_h, self.like.d_d, self.packed)


class HetGroup:
    def __init__(self, het, walkers, t_obs_start=0.0, t_obs_end=1.0):
        t = torch()
        self.het = het
        self.params = t.as_tensor(walkers, dtype=t.float64, device=device()).contiguous()
        self.t_obs_start, self.t_obs_end = t_obs_start, t_obs_end
        self.flags = t.zeros(3, dtype=t.int32, device=device())

    @property
    def size(self):
        return self.params.shape[1]

    def source(self, precision="fp64"):
        """Descriptor of this group for bbhx_uneven_batch: the walkers' parameters and the
        device buffers the batch fills (PhenomHM records, observation limits, sums); no host
        synchronisation."""
        from .waveforms.ringdownphenomd import dspin

        t = torch()
        het = self.het
        gen = het.template_gen
        ap, rg = gen.amp_phase_gen, gen.response_gen
        ells, mms = ap.mode_tensors(None)
        B, M, L = self.size, int(ells.numel()), int(het.freqs.numel())
        f64 = dict(dtype=t.float64, device=device())
        nbytes = int(_lib.lib().bbhx_mode_coeffs_bytes())
        coeffs = t.empty(B * M * nbytes, dtype=t.uint8, device=device())
        ts, te = t.empty(B, **f64), t.empty(B, **f64)
        self.d_h = t.empty(B, dtype=t.complex128, device=device())
        self.h_h = t.empty(B, dtype=t.complex128, device=device())
        self.packed = t.empty(3 * B, **f64)
        tab = ap.qnm_table
        self._keep = (coeffs, ts, te, ells, mms, tab)
        p = lambda a: _lib.dptr(a).value  # noqa: E731
        row = lambda k: self.params.data_ptr() + 8 * k * B  # noqa: E731
        group = HdynGroupC(
            orbits=rg.orbit_handle.ptr.value, d_h=p(self.d_h), h_h=p(self.h_h), coeffs=p(coeffs),
            ells=p(ells), mms=p(mms), phi_ref=row(5), inc=row(7), lam=row(8), beta=row(9),
            psi=row(10), t_ref=row(11), t_init=float(ap.initial_t_val), t_start=p(ts), t_end=p(te),
            freqs=p(het.freqs), h0=p(het._h0_flat), consts=p(het.data_constants),
            TDItag=rg.TDItag_int, rescaled=int(rg.rescaled), tdi2=int(rg.tdi2), num_modes=M,
            length=L, num_bin_all=B)
        return HdynSourceC(group=group, params=p(self.params), qnm_table=p(tab),
                           qnm_n=int(tab.shape[1]), dspin=float(dspin),
                           t_obs_start_L=float(self.t_obs_start * YRSID_SI),
                           t_obs_end_L=float(self.t_obs_end * YRSID_SI),
                           run_phenomd=int(ap.run_phenomd), flags=p(self.flags))

    def lnl(self):
        return pack_lnl(self.d_h, self.h_h, self.het.reference_d_d, self.packed)


class Autotuner:
    """Times the persistent kernel's launch shapes on a prepared batch and keeps the fastest
    per batch signature (in memory; ``table`` can be saved / preloaded by the caller)."""

    TILES = (1024, 2048, 4096)
    CTAS = (2, 3, 4, 8)

    def __init__(self, table=None, repeats=2):
        self.table = dict(table or {})
        self.repeats = repeats

    @staticmethod
    def signature(descs, hdescs, precision):
        return (precision, len(descs), sum(d.num_bin_all for d in descs),
                max((d.data_length for d in descs), default=0),
                max((d.length for d in descs), default=0), len(hdescs),
                sum(h.group.num_bin_all for h in hdescs),
                max((h.group.length for h in hdescs), default=0))

    def best(self, descs, hdescs, precision, launch):
        key = self.signature(descs, hdescs, precision)
        if key in self.table:
            return self.table[key]
        t = torch()
        timings = {}
        for tile, ctas in itertools.product(self.TILES, self.CTAS):
            launch(tile, ctas)  # warm-up of this shape
            e0 = t.cuda.Event(enable_timing=True)
            e1 = t.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(self.repeats):
                launch(tile, ctas)
            e1.record()
            e1.synchronize()
            timings[(tile, ctas)] = e0.elapsed_time(e1) / self.repeats
        choice = min(timings, key=timings.get)
        self.table[key] = choice
        self.last_timings = timings
        return choice


# Mixed form of a direct group: its FP32 amplitude / transfer cubics are evaluated across a
# whole spline segment, and with coarse sparse grids over long data streams a segment spans
# ~1e4 data bins; the FP32 rounding of the cubic, largest relative to the template where the
# transfer functions pass near the TDI zeros (and the weights are largest), then reaches
# ~1e-5 <h|h> in lnL.  Groups whose segments span more data bins per knot interval than this
# run in FP64 (a second persistent launch) when the batch is mixed.
MIXED_MAX_BINS_PER_KNOT = 2048


class UnevenBatch:
    def __init__(self, direct_groups=(), het_groups=(), precision="mixed", autotuner=None,
                 shape=None, mixed_max_bins_per_knot=MIXED_MAX_BINS_PER_KNOT):
        self.direct = list(direct_groups)
        self.het = list(het_groups)
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}, got {precision!r}")
        self.precision = precision
        self.mixed_max_bins_per_knot = mixed_max_bins_per_knot
        self.autotuner = autotuner if autotuner is not None else Autotuner()
        # launch shape per precision class, {"fp64" | "mixed": (tile_bins, ctas_per_sm)};
        # a missing entry is autotuned on the first run
        self.shape = dict(shape or {})
        self.graph = None
        if len(self.direct) > 64 or len(self.het) > 64:
            raise ValueError("at most 64 direct and 64 heterodyned groups per batch")

    def group_precisions(self):
        """Arithmetic of every group (direct groups first): a mixed batch runs the direct
        groups whose segments span more than mixed_max_bins_per_knot data bins in FP64."""
        out = []
        for g in self.direct:
            coarse = int(g.like.data_freqs.numel()) / g.length > self.mixed_max_bins_per_knot
            out.append("fp64" if (self.precision == "fp64" or coarse) else "mixed")
        return out + [self.precision] * len(self.het)

    def _launch(self, descs, hdescs, precision, tile, ctas):
        arr = (DirectSourceC * max(len(descs), 1))(*descs)
        harr = (HdynSourceC * max(len(hdescs), 1))(*hdescs)
        _lib.call("bbhx_uneven_batch", ctypes.cast(arr, ctypes.c_void_p), len(descs),
                  ctypes.cast(harr, ctypes.c_void_p), len(hdescs), PRECISIONS[precision],
                  int(tile), int(ctas), _lib.stream())

    def run(self):
        """All groups' lnL (list of device tensors, direct groups first).  The groups of each
        precision class run as one call: one launch builds every direct group's sparse grids
        and splines, one persistent launch evaluates every direct tile and heterodyned walker."""
        precs = self.group_precisions()
        classes = {}
        for g, pr in zip(self.direct, precs):
            classes.setdefault(pr, ([], []))[0].append(g.source(pr))
        for h, pr in zip(self.het, precs[len(self.direct):]):
            classes.setdefault(pr, ([], []))[1].append(h.source(pr))
        for pr, (descs, hdescs) in classes.items():
            if pr not in self.shape:
                self.shape[pr] = self.autotuner.best(
                    descs, hdescs, pr, lambda tl, c: self._launch(descs, hdescs, pr, tl, c))
            self._launch(descs, hdescs, pr, *self.shape[pr])
        return [g.lnl() for g in self.direct] + [h.lnl() for h in self.het]

    def capture(self):
        """Record run() in a CUDA graph (after one eager run that also autotunes), execute it
        once and return the output tensors (refreshed in place by every replay())."""
        t = torch()
        self.run()
        t.cuda.synchronize()
        s = t.cuda.Stream()
        s.wait_stream(t.cuda.current_stream())
        with t.cuda.stream(s):
            self.run()  # warm the allocator on the capture stream
        t.cuda.current_stream().wait_stream(s)
        t.cuda.synchronize()
        self.graph = t.cuda.CUDAGraph()
        with t.cuda.graph(self.graph):
            self.outputs = self.run()
        self.graph.replay()  # capturing records the work; this executes it once
        return self.outputs

    def set_params(self, group_index, params):
        """Copy new parameters into a group's (graph-captured) parameter tensor."""
        groups = self.direct + self.het
        groups[group_index].params.copy_(torch().as_tensor(params, dtype=torch().float64))

    def replay(self):
        self.graph.replay()
        return self.outputs

    def flags(self):
        """Device error flags of every group (window search, orbit coverage, spins)."""
        return [g.flags for g in self.direct + self.het]
