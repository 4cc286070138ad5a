"""simcore_b200: B200 Brownian-dynamics step for semiflexible filaments.

Python binding of the C ABI in include/simcore_gpu.h (libsimcore_b200.so,
built in-tree by simcore_b200/build.py).  The library is required: importing
this package on a machine where it was not built raises, and every compute
call runs the CUDA kernels -- there is no CPU fallback.

    ctx = Context(system, filaments, sites, precision="fp64")
    ctx.step(2)              # two reference steps (one midpoint BD step)
    xyz = ctx.sites()
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsimcore_b200.so")

SC_OK = 0
STATUS_NAMES = {0: "SC_OK", 1: "SC_ERR_INVALID_ARG", 2: "SC_ERR_OOM", 3: "SC_ERR_NAN",
                4: "SC_ERR_LIST_OVERFLOW", 5: "SC_ERR_TIMEOUT", 6: "SC_ERR_CUDA",
                7: "SC_ERR_UNPHYSICAL", 8: "SC_ERR_INSERTION", 9: "SC_ERR_NO_DEVICE"}
PRECISION = {"fp64": 0, "mixed": 1}

# Every symbol include/simcore_gpu.h declares.
EXPORTED = ["sc_create", "sc_destroy", "sc_last_error", "sc_add_filaments",
            "sc_filament_n_bonds", "sc_interact", "sc_update_positions", "sc_step",
            "sc_step_graph", "sc_synchronize", "sc_get_sites", "sc_set_sites",
            "sc_get_prev_sites", "sc_get_random_forces", "sc_get_bond_forces",
            "sc_get_bond_geometry", "sc_set_capture", "sc_get_site_forces",
            "sc_get_tensions", "sc_get_filament_state", "sc_get_dr_tot", "sc_get_pairs",
            "sc_get_bond_cells", "sc_get_counters", "sc_get_stream", "sc_set_kernel_timing",
            "sc_get_kernel_timing", "sc_get_graph_time", "sc_set_fast_integrator",
            "sc_pair_forces_noalloc", "sc_insert_filaments", "sc_add_crosslinks",
            "sc_get_crosslink_forces", "sc_set_integrator_layout", "sc_autotune",
            "sc_add_replicas", "sc_get_replica_counters", "sc_checkpoint", "sc_restore",
            "sc_set_noise_key", "sc_output_open", "sc_output_write", "sc_output_close",
            "sc_analysis_sample", "sc_analysis_results", "sc_global_order",
            "sc_set_thermo", "sc_thermo_open", "sc_get_thermo", "sc_get_potential_energy",
            "sc_set_exact_near_parallel", "sc_set_near_parallel_threshold",
            "sc_set_fused_pairs", "sc_diffusion_init",
            "sc_diffusion_sample", "sc_diffusion_results", "sc_insert_filaments_gpu"]


class ScError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (STATUS_NAMES.get(code, code), msg))
        self.code = code


class SystemDesc(ctypes.Structure):
    _fields_ = [("n_dim", ctypes.c_int), ("system_radius", ctypes.c_double),
                ("delta", ctypes.c_double), ("wca_eps", ctypes.c_double),
                ("wca_sig", ctypes.c_double), ("f_cutoff", ctypes.c_double),
                ("stoch_flag", ctypes.c_int), ("interaction_flag", ctypes.c_int),
                ("like_like_interactions", ctypes.c_int), ("seed", ctypes.c_uint32),
                ("precision", ctypes.c_int), ("device", ctypes.c_int)]


class FilamentParams(ctypes.Structure):
    _fields_ = [("length", ctypes.c_double), ("persistence_length", ctypes.c_double),
                ("diameter", ctypes.c_double), ("min_bond_length", ctypes.c_double),
                ("friction_ratio", ctypes.c_double)]


class Counters(ctypes.Structure):
    _fields_ = [("i_step", ctypes.c_int64), ("n_rebuilds", ctypes.c_int64),
                ("n_pairs", ctypes.c_int64), ("pair_capacity", ctypes.c_int64),
                ("n_filaments", ctypes.c_int64), ("n_sites", ctypes.c_int64),
                ("n_bonds", ctypes.c_int64), ("n_cells_1d", ctypes.c_int32),
                ("cell_length", ctypes.c_double), ("dr_update", ctypes.c_double),
                ("kernel_launches", ctypes.c_int64), ("n_replicas", ctypes.c_int32),
                ("n_list_regrowths", ctypes.c_int64)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError("simcore_b200: %s is not built (run simcore_b200/build.py); "
                          "there is no CPU fallback" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    lib.sc_last_error.restype = ctypes.c_char_p
    lib.sc_last_error.argtypes = [vp]
    lib.sc_get_stream.restype = vp
    lib.sc_get_stream.argtypes = [vp]
    for name in EXPORTED:
        fn = getattr(lib, name)
        if name not in ("sc_last_error", "sc_get_stream"):
            fn.restype = ctypes.c_int
    return lib


lib = _load()


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def filament_n_bonds(params):
    fp = FilamentParams(**params)
    return lib.sc_filament_n_bonds(ctypes.byref(fp))


INSERTION = {"random": 0, "random_nematic": 1, "random_polar": 2}


def insert_filaments(n_dim, system_radius, seed, n_bonds, lengths, persistence_lengths,
                     diameter=1.0, max_attempts=10000, insertion="random", device=None):
    """Seeded random insertion with overlap rejection.  Returns sites.  With
    a device, the overlap tests run on that GPU (sc_insert_filaments_gpu);
    the result is the same, bit for bit."""
    n_bonds = np.ascontiguousarray(n_bonds, dtype=np.int32)
    lengths = np.ascontiguousarray(lengths, dtype=np.float64)
    lps = np.ascontiguousarray(persistence_lengths, dtype=np.float64)
    xyz = np.zeros((int(np.sum(n_bonds + 1)), 3))
    args = (ctypes.c_int(n_dim), ctypes.c_double(system_radius), ctypes.c_uint64(seed),
            ctypes.c_int(len(n_bonds)), _p(n_bonds), _p(lengths), _p(lps),
            ctypes.c_double(diameter), ctypes.c_int(INSERTION[insertion]),
            ctypes.c_int(max_attempts), _p(xyz))
    if device is None:
        rc = lib.sc_insert_filaments(*args)
    else:
        rc = lib.sc_insert_filaments_gpu(ctypes.c_int(device), *args)
    if rc != SC_OK:
        raise ScError(rc, "random insertion failed")
    return xyz


class Context:
    """One simulated system on one GPU (an sc_ctx)."""

    def __init__(self, system, filaments, sites, precision="fp64", device=0, replicas=None):
        """replicas: None for one system, or a list of dicts (system_radius,
        seed, n_filaments) of independent systems whose filaments and sites
        follow one another in `filaments` and `sites`."""
        desc = SystemDesc(n_dim=system["n_dim"], system_radius=system["system_radius"],
                          delta=system["delta"], wca_eps=system.get("wca_eps", 1.0),
                          wca_sig=system.get("wca_sig", 1.0),
                          f_cutoff=system.get("f_cutoff", 2000.0),
                          stoch_flag=system.get("stoch_flag", 1),
                          interaction_flag=system.get("interaction_flag", 1),
                          like_like_interactions=system.get("like_like_interactions", 1),
                          seed=system.get("seed", 0), precision=PRECISION[precision],
                          device=device)
        h = ctypes.c_void_p()
        rc = lib.sc_create(ctypes.byref(desc), ctypes.byref(h))
        if rc != SC_OK:
            raise ScError(rc, "sc_create failed")
        self.h = h
        self.n_dim = system["n_dim"]
        fils = (FilamentParams * len(filaments))(*[FilamentParams(**f) for f in filaments])
        sites = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
        if replicas is None:
            self._check(lib.sc_add_filaments(h, ctypes.c_int(len(filaments)), fils, _p(sites),
                                             ctypes.c_int64(sites.shape[0])))
        else:
            radius = np.array([r["system_radius"] for r in replicas], dtype=np.float64)
            seeds = np.array([r["seed"] for r in replicas], dtype=np.uint32)
            nfil = np.array([r["n_filaments"] for r in replicas], dtype=np.int32)
            self._check(lib.sc_add_replicas(h, ctypes.c_int(len(replicas)), _p(radius),
                                            _p(seeds), _p(nfil), ctypes.c_int(len(filaments)),
                                            fils, _p(sites), ctypes.c_int64(sites.shape[0])))
        self.n_replicas = 1 if replicas is None else len(replicas)
        c = self.counters()
        self.n_sites, self.n_bonds, self.n_fil = c.n_sites, c.n_bonds, c.n_filaments

    def _check(self, rc):
        if rc != SC_OK:
            msg = lib.sc_last_error(self.h)
            raise ScError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "h", None):
            lib.sc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # stepping
    def step(self, n=1):
        self._check(lib.sc_step(self.h, ctypes.c_int(n)))

    def step_graph(self, n=1):
        self._check(lib.sc_step_graph(self.h, ctypes.c_int(n)))

    def add_crosslinks(self, site_a, site_b, k_spring=10.0, k_spring_compress=-1.0,
                       rest_length=0.0):
        """Static doubly-bound tethers between global site indices."""
        a = np.ascontiguousarray(site_a, dtype=np.int32)
        b = np.ascontiguousarray(site_b, dtype=np.int32)
        if a.shape != b.shape:
            raise ValueError("site_a and site_b differ in length")
        self.n_links = int(a.size)
        self._check(lib.sc_add_crosslinks(self.h, ctypes.c_int(a.size), _p(a), _p(b),
                                          ctypes.c_double(k_spring),
                                          ctypes.c_double(k_spring_compress),
                                          ctypes.c_double(rest_length)))

    def crosslink_forces(self):
        f = np.zeros((getattr(self, "n_links", 0), 3))
        self._check(lib.sc_get_crosslink_forces(self.h, _p(f)))
        return f

    def interact(self):
        self._check(lib.sc_interact(self.h))

    def update_positions(self):
        self._check(lib.sc_update_positions(self.h))

    def synchronize(self):
        self._check(lib.sc_synchronize(self.h))

    def set_fast_integrator(self, on=True):
        self._check(lib.sc_set_fast_integrator(self.h, ctypes.c_int(1 if on else 0)))

    def set_integrator_layout(self, warp_max_sites=32, block_sites=0):
        """Filaments of at most warp_max_sites sites on the warp-synchronous
        integrator (0: none), the rest on blocks of block_sites sites."""
        self._check(lib.sc_set_integrator_layout(self.h, ctypes.c_int(warp_max_sites),
                                                 ctypes.c_int(block_sites)))

    def autotune(self, cache_path=None):
        """Times the integrator layouts on this context's state (restored
        afterwards), applies the fastest; returns (warp_max_sites,
        block_sites).  cache_path: optional text cache keyed by shape."""
        w = ctypes.c_int()
        b = ctypes.c_int()
        path = cache_path.encode() if cache_path else None
        self._check(lib.sc_autotune(self.h, path, ctypes.byref(w), ctypes.byref(b)))
        return w.value, b.value

    def set_capture(self, on=True):
        self._check(lib.sc_set_capture(self.h, ctypes.c_int(1 if on else 0)))

    @property
    def stream(self):
        return lib.sc_get_stream(self.h)

    # state
    def _vec(self, fn, n, out=None):
        if out is None:
            a = np.zeros((n, 3))
        else:
            a = out
            if a.shape != (n, 3) or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("out must be a C-contiguous float64 array of shape (%d, 3)" % n)
        self._check(fn(self.h, _p(a)))
        return a

    def sites(self, out=None):
        """Site positions (N_s x 3).  out: an array to fill instead (a pinned
        host buffer makes the copy run at full link speed)."""
        return self._vec(lib.sc_get_sites, self.n_sites, out)

    def set_sites(self, xyz):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        self._check(lib.sc_set_sites(self.h, _p(xyz)))

    def prev_sites(self):
        return self._vec(lib.sc_get_prev_sites, self.n_sites)

    def random_forces(self):
        return self._vec(lib.sc_get_random_forces, self.n_sites)

    def site_forces(self):
        return self._vec(lib.sc_get_site_forces, self.n_sites)

    def bond_forces(self):
        f = np.zeros((self.n_bonds, 3))
        t = np.zeros((self.n_bonds, 3))
        self._check(lib.sc_get_bond_forces(self.h, _p(f), _p(t)))
        return f, t

    def bond_geometry(self):
        pos = np.zeros((self.n_bonds, 3))
        spos = np.zeros((self.n_bonds, 3))
        u = np.zeros((self.n_bonds, 3))
        ln = np.zeros(self.n_bonds)
        self._check(lib.sc_get_bond_geometry(self.h, _p(pos), _p(spos), _p(u), _p(ln)))
        return pos, spos, u, ln

    def tensions(self):
        a = np.zeros(self.n_bonds)
        self._check(lib.sc_get_tensions(self.h, _p(a)))
        return a

    def filament_state(self):
        sw = np.zeros(self.n_fil, dtype=np.int32)
        nn = np.zeros(self.n_fil, dtype=np.int32)
        self._check(lib.sc_get_filament_state(self.h, _p(sw), _p(nn)))
        return sw, nn

    def dr_tot(self):
        a = np.zeros(self.n_sites)
        self._check(lib.sc_get_dr_tot(self.h, _p(a)))
        return a

    def pairs(self):
        n = ctypes.c_int64()
        self._check(lib.sc_get_pairs(self.h, None, ctypes.c_int64(0), ctypes.byref(n)))
        out = np.zeros((max(n.value, 1), 2), dtype=np.int32)
        self._check(lib.sc_get_pairs(self.h, _p(out), ctypes.c_int64(n.value), ctypes.byref(n)))
        return out[:n.value]

    def bond_cells(self):
        a = np.zeros((self.n_bonds, 3), dtype=np.int32)
        self._check(lib.sc_get_bond_cells(self.h, _p(a)))
        return a

    def set_kernel_timing(self, on=True):
        self._check(lib.sc_set_kernel_timing(self.h, ctypes.c_int(1 if on else 0)))

    def kernel_timing(self):
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        self._check(lib.sc_get_kernel_timing(self.h, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def graph_time_ms(self):
        ms = ctypes.c_double()
        self._check(lib.sc_get_graph_time(self.h, ctypes.byref(ms)))
        return ms.value

    def checkpoint(self):
        """The whole simulation state as bytes (sc_checkpoint)."""
        size = ctypes.c_size_t()
        self._check(lib.sc_checkpoint(self.h, None, ctypes.c_size_t(0), ctypes.byref(size)))
        buf = ctypes.create_string_buffer(size.value)
        self._check(lib.sc_checkpoint(self.h, buf, size, ctypes.byref(size)))
        return buf.raw

    def restore(self, data):
        """Loads a checkpoint of a context holding the same systems."""
        self._check(lib.sc_restore(self.h, ctypes.c_char_p(data), ctypes.c_size_t(len(data))))

    def set_noise_key(self, seed, replica=-1):
        self._check(lib.sc_set_noise_key(self.h, ctypes.c_int(replica), ctypes.c_uint32(seed)))

    def output_open(self, run_name, n_steps, n_posit=0, n_spec=0, species_name="filament"):
        """Reference-format spec/posit files (<run>_filament_<species>.spec /
        .posit); write frames with output_write() after every step."""
        self._check(lib.sc_output_open(self.h, run_name.encode(), species_name.encode(),
                                       ctypes.c_int(n_steps), ctypes.c_int(n_posit),
                                       ctypes.c_int(n_spec)))

    def output_write(self):
        self._check(lib.sc_output_write(self.h))

    def output_close(self):
        self._check(lib.sc_output_close(self.h))

    def analysis_sample(self, n_bins=100):
        self._check(lib.sc_analysis_sample(self.h, ctypes.c_int(n_bins)))

    def analysis_results(self, n_bins=100):
        """(mse2e, mse2e_err, n_samples, theta_hist[nrep, max_joints, n_bins])."""
        R = self.n_replicas
        m = np.zeros(R)
        e = np.zeros(R)
        ns = ctypes.c_int64()
        mj = ctypes.c_int32()
        self._check(lib.sc_analysis_results(self.h, None, None, ctypes.byref(ns),
                                            ctypes.byref(mj), None))
        hist = np.zeros((R, max(mj.value, 1), n_bins), dtype=np.int64)
        self._check(lib.sc_analysis_results(self.h, _p(m), _p(e), ctypes.byref(ns),
                                            ctypes.byref(mj), _p(hist)))
        return m, e, ns.value, hist

    def global_order(self):
        R = self.n_replicas
        p = np.zeros((R, 3))
        q = np.zeros((R, 9))
        self._check(lib.sc_global_order(self.h, _p(p), _p(q)))
        return p, q

    def diffusion_init(self, interval):
        """Centre-of-mass diffusion analysis: current filament averages as
        time origins, windows of `interval` samples."""
        self._check(lib.sc_diffusion_init(self.h, int(interval)))
        self._dif_interval = int(interval)

    def diffusion_sample(self):
        self._check(lib.sc_diffusion_sample(self.h))

    def diffusion_results(self):
        """(msd, msd_err, vcf, vcf_err), each (systems, interval); a single
        system's arrays drop the systems axis."""
        R, T = self.n_replicas, self._dif_interval
        out = [np.zeros((R, T)) for _ in range(4)]
        self._check(lib.sc_diffusion_results(self.h, *[_p(a) for a in out]))
        return tuple(a[0] for a in out) if R == 1 else tuple(out)

    def set_exact_near_parallel(self, on=True):
        """Mixed precision: nearly parallel pairs evaluated from the FP64 sites."""
        self._check(lib.sc_set_exact_near_parallel(self.h, 1 if on else 0))

    def set_near_parallel_threshold(self, s2):
        """Mixed precision: |u1 x u2|^2 below which side-by-side pairs are FP64."""
        self._check(lib.sc_set_near_parallel_threshold(self.h, ctypes.c_double(s2)))

    def set_fused_pairs(self, on=True):
        """Fast mixed precision: the integrator evaluates the pairs itself (no
        pair stage), with the same bits."""
        self._check(lib.sc_set_fused_pairs(self.h, 1 if on else 0))

    def set_thermo(self, n_thermo):
        """Pair virial sums every step and a pressure record every n_thermo
        steps (0: off)."""
        self._check(lib.sc_set_thermo(self.h, int(n_thermo)))

    def thermo_open(self, run_name, n_steps):
        """Writes the records from now on to <run_name>.thermo."""
        self._check(lib.sc_thermo_open(self.h, run_name.encode(), int(n_steps)))

    def thermo_records(self, max_records=100000):
        """(i_step (k), pressure tensor (k, systems, 9), pressure (k, systems),
        volume (k, systems)) of the records since the last call; a single
        system's arrays drop the systems axis."""
        R = self.n_replicas
        st = np.zeros(max_records, dtype=np.int64)
        P = np.zeros((max_records, R, 9))
        p = np.zeros((max_records, R))
        V = np.zeros((max_records, R))
        n = ctypes.c_int(0)
        self._check(lib.sc_get_thermo(self.h, int(max_records), ctypes.byref(n), _p(st), _p(P),
                                      _p(p), _p(V)))
        k = n.value
        if R == 1:
            return st[:k], P[:k, 0], p[:k, 0], V[:k, 0]
        return st[:k], P[:k], p[:k], V[:k]

    def potential_energy(self):
        """Potential energy of every filament of the last pair stage."""
        out = np.zeros(self.n_fil)
        self._check(lib.sc_get_potential_energy(self.h, _p(out)))
        return out

    def replica_counters(self):
        """(rebuilds, pairs) per system."""
        nr = np.zeros(self.n_replicas, dtype=np.int64)
        npr = np.zeros(self.n_replicas, dtype=np.int64)
        self._check(lib.sc_get_replica_counters(self.h, _p(nr), _p(npr)))
        return nr, npr

    def counters(self):
        c = Counters()
        self._check(lib.sc_get_counters(self.h, ctypes.byref(c)))
        return c
