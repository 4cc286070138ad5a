"""ctypes bindings of the CPU checkers (test infrastructure).

Two libraries with one interface:
  Oracle    -- oracle/libscoracle.so, the plain-C restatement of the path;
  Reference -- oracle/_ref/libscref.so, the reference's own hot-path sources
               driven by a harness (built only where the reference tree is
               present; absent otherwise).
Both take the same system/filament descriptors and site positions and expose
the same getters, so a test can run either, or both, on one configuration.
"""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "libscoracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libscref.so")


class SystemDesc(ctypes.Structure):
    _fields_ = [("n_dim", ctypes.c_int), ("system_radius", ctypes.c_double),
                ("delta", ctypes.c_double), ("wca_eps", ctypes.c_double),
                ("wca_sig", ctypes.c_double), ("f_cutoff", ctypes.c_double),
                ("stoch_flag", ctypes.c_int), ("interaction_flag", ctypes.c_int),
                ("like_like_interactions", ctypes.c_int), ("seed", ctypes.c_uint),
                ("n_threads", ctypes.c_int)]


class FilamentDesc(ctypes.Structure):
    _fields_ = [("length", ctypes.c_double), ("persistence_length", ctypes.c_double),
                ("diameter", ctypes.c_double), ("min_bond_length", ctypes.c_double),
                ("friction_ratio", ctypes.c_double)]


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class _Checker:
    prefix = None
    so = None

    def __init__(self, system, filaments, sites, n_threads=1):
        self.lib = ctypes.CDLL(self.so)
        p = self.prefix
        L = self.lib
        getattr(L, p + "create").restype = ctypes.c_void_p
        getattr(L, p + "create").argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_int]
        for name in ("n_sites", "n_bonds", "n_cells_1d", "i_step"):
            getattr(L, p + name).restype = ctypes.c_int
            getattr(L, p + name).argtypes = [ctypes.c_void_p]
        for name in ("cell_length", "dr_update"):
            getattr(L, p + name).restype = ctypes.c_double
            getattr(L, p + name).argtypes = [ctypes.c_void_p]
        getattr(L, p + "n_rebuilds").restype = ctypes.c_long
        getattr(L, p + "n_rebuilds").argtypes = [ctypes.c_void_p]
        getattr(L, p + "get_pairs").restype = ctypes.c_long
        getattr(L, p + "get_pairs").argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long]
        getattr(L, p + "destroy").argtypes = [ctypes.c_void_p]
        defaults = dict(wca_eps=1.0, wca_sig=1.0, f_cutoff=2000.0, stoch_flag=1,
                        interaction_flag=1, like_like_interactions=1, seed=0)
        vals = dict(defaults, **system)
        sysd = SystemDesc(**{k: vals[k] for k, _ in SystemDesc._fields_ if k != "n_threads"},
                          n_threads=n_threads)
        fils = (FilamentDesc * len(filaments))(*[FilamentDesc(**f) for f in filaments])
        sites = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
        self.h = getattr(L, p + "create")(ctypes.byref(sysd), len(filaments), fils,
                                          _ptr(sites), sites.shape[0])
        if not self.h:
            raise RuntimeError("%screate failed" % p)
        self.n_sites = getattr(L, p + "n_sites")(self.h)
        self.n_bonds = getattr(L, p + "n_bonds")(self.h)
        self.n_fil = len(filaments)

    def _call(self, name, *args):
        return getattr(self.lib, self.prefix + name)(ctypes.c_void_p(self.h), *args)

    def close(self):
        if self.h:
            self._call("destroy")
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n_cells_1d(self):
        return self._call("n_cells_1d")

    @property
    def cell_length(self):
        return self._call("cell_length")

    @property
    def dr_update(self):
        return self._call("dr_update")

    @property
    def n_rebuilds(self):
        return self._call("n_rebuilds")

    @property
    def i_step(self):
        return self._call("i_step")

    def sites(self):
        a = np.zeros((self.n_sites, 3))
        self._call("get_sites", _ptr(a))
        return a

    def prev_sites(self):
        a = np.zeros((self.n_sites, 3))
        self._call("get_prev_sites", _ptr(a))
        return a

    def site_forces(self):
        a = np.zeros((self.n_sites, 3))
        self._call("get_site_forces", _ptr(a))
        return a

    def random_forces(self):
        a = np.zeros((self.n_sites, 3))
        self._call("get_random_forces", _ptr(a))
        return a

    def bond_forces(self):
        f = np.zeros((self.n_bonds, 3))
        t = np.zeros((self.n_bonds, 3))
        self._call("get_bond_ft", _ptr(f), _ptr(t))
        return f, t

    def tensions(self):
        a = np.zeros(self.n_bonds)
        self._call("get_tensions", _ptr(a))
        return a

    def bond_geometry(self):
        pos = np.zeros((self.n_bonds, 3))
        spos = np.zeros((self.n_bonds, 3))
        u = np.zeros((self.n_bonds, 3))
        ln = np.zeros(self.n_bonds)
        self._call("get_bond_geom", _ptr(pos), _ptr(spos), _ptr(u), _ptr(ln))
        return pos, spos, u, ln

    def filament_state(self):
        sw = np.zeros(self.n_fil, dtype=np.int32)
        nn = np.zeros(self.n_fil, dtype=np.int32)
        self._call("get_filament_state", _ptr(sw), _ptr(nn))
        return sw, nn

    def pairs(self):
        n = self._call("get_pairs", None, ctypes.c_long(0))
        out = np.zeros((max(n, 1), 2), dtype=np.int32)
        self._call("get_pairs", _ptr(out), ctypes.c_long(n))
        return out[:n]

    def bond_cells(self):
        a = np.zeros((self.n_bonds, 3), dtype=np.int32)
        self._call("get_bond_cells", _ptr(a))
        return a

    def dr_tot(self):
        a = np.zeros(self.n_sites)
        self._call("get_dr_tot", _ptr(a))
        return a

    def set_thermo(self, n_thermo):
        self._call("set_thermo", ctypes.c_int(n_thermo))

    def thermo_records(self, max_records=100000):
        """(i_step, pressure tensor (k, 9), pressure, volume) of the records
        taken since the last call."""
        getattr(self.lib, self.prefix + "thermo_records").restype = ctypes.c_long
        st = np.zeros(max_records, dtype=np.int64)
        P = np.zeros((max_records, 9))
        p = np.zeros(max_records)
        V = np.zeros(max_records)
        n = self._call("thermo_records", ctypes.c_long(max_records), _ptr(st), _ptr(P), _ptr(p),
                       _ptr(V))
        return st[:n], P[:n], p[:n], V[:n]

    def stress(self):
        a = np.zeros(9)
        self._call("get_stress", _ptr(a))
        return a

    def potential_energy(self):
        a = np.zeros(self.n_fil)
        self._call("get_potential_energy", _ptr(a))
        return a


class Oracle(_Checker):
    """The plain-C restatement (always available once built)."""
    prefix = "sco_"
    so = ORACLE_SO

    def step(self, n=1):
        self.lib.sco_step.restype = ctypes.c_int
        rc = self._call("step", ctypes.c_int(n))
        if rc != 0:
            raise RuntimeError("oracle step failed (unphysical displacement)")

    def set_sites(self, xyz):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        self._call("set_sites", _ptr(xyz))

    def add_crosslinks(self, site_a, site_b, k_spring=10.0, k_spring_compress=-1.0,
                       rest_length=0.0):
        a = np.ascontiguousarray(site_a, dtype=np.int32)
        b = np.ascontiguousarray(site_b, dtype=np.int32)
        self.n_links = int(a.size)
        self.lib.sco_add_crosslinks.restype = ctypes.c_int
        rc = self._call("add_crosslinks", ctypes.c_int(a.size), _ptr(a), _ptr(b),
                        ctypes.c_double(k_spring), ctypes.c_double(k_spring_compress),
                        ctypes.c_double(rest_length))
        if rc != 0:
            raise RuntimeError("oracle rejected the crosslinks")

    def crosslink_forces(self):
        f = np.zeros((getattr(self, "n_links", 0), 3))
        self._call("get_crosslink_forces", _ptr(f))
        return f

    def frictions(self):
        out = [np.zeros(self.n_fil) for _ in range(4)]
        self._call("get_frictions", *[_ptr(a) for a in out])
        return out


class Reference(_Checker):
    """The reference's own code (oracle/_ref), where it was built."""
    prefix = "scref_"
    so = REF_SO

    @staticmethod
    def available():
        return os.path.exists(REF_SO)

    def step(self, n=1):
        self.lib.scref_step.restype = ctypes.c_double
        t = self._call("step", ctypes.c_int(n))
        if t < 0:
            raise RuntimeError("reference step failed (unphysical displacement)")
        return t

    def frictions(self):
        out = [np.zeros(self.n_fil) for _ in range(4)]
        self._call("get_frictions", *[_ptr(a) for a in out])
        return out

    def add_crosslinks(self, site_a, site_b, k_spring=10.0, k_spring_compress=-1.0,
                       rest_length=0.0):
        """Doubly-bound crosslinks made and attached by the reference's own
        Crosslink and Anchor code (zero unbinding rate, no diffusion)."""
        a = np.ascontiguousarray(site_a, dtype=np.int32)
        b = np.ascontiguousarray(site_b, dtype=np.int32)
        self.n_links = int(a.size)
        self.lib.scref_add_crosslinks.restype = ctypes.c_int
        rc = self._call("add_crosslinks", ctypes.c_int(a.size), _ptr(a), _ptr(b),
                        ctypes.c_double(k_spring), ctypes.c_double(k_spring_compress),
                        ctypes.c_double(rest_length))
        if rc != 0:
            raise RuntimeError("reference rejected the crosslinks")

    def crosslink_forces(self):
        f = np.zeros((getattr(self, "n_links", 0), 3))
        self._call("get_crosslink_forces", _ptr(f))
        return f

    def analysis_sample(self, n_bins=100):
        """FilamentSpecies::RunMse2eAnalysis + RunThetaAnalysis, as the
        reference runs them after a step."""
        self._call("analysis_sample", ctypes.c_int(n_bins))
        self._n_bins = n_bins

    def analysis_results(self):
        """(mse2e mean, its error, samples, histogram (joints, bins))."""
        m, e = ctypes.c_double(), ctypes.c_double()
        n, j = ctypes.c_long(), ctypes.c_int()
        self._call("analysis_results", ctypes.byref(m), ctypes.byref(e), ctypes.byref(n),
                   ctypes.byref(j), None)
        hist = np.zeros((j.value, self._n_bins), dtype=np.int64)
        self._call("analysis_results", None, None, None, None, _ptr(hist))
        return m.value, e.value, n.value, hist

    def diffusion_init(self, interval):
        self._call("diffusion_init", ctypes.c_int(interval))
        self._dif_interval = interval

    def diffusion_sample(self):
        self._call("diffusion_sample")

    def diffusion_results(self):
        out = [np.zeros(self._dif_interval) for _ in range(4)]
        self._call("diffusion_results", *[_ptr(a) for a in out])
        return tuple(out)

    def write_spec_frame(self, path):
        """Appends one spec frame, written by the reference's own writers."""
        if self._call("write_spec_frame", ctypes.c_char_p(path.encode())) != 0:
            raise RuntimeError("spec frame not written")

    def write_posit_frame(self, path):
        """Appends one posit frame, written by the reference's own writers."""
        if self._call("write_posit_frame", ctypes.c_char_p(path.encode())) != 0:
            raise RuntimeError("posit frame not written")

    def global_order(self):
        """Polar order vector (3) and nematic tensor (3 x 3) of the current
        state, as the reference's first global-order sample."""
        polar, nem = np.zeros(3), np.zeros(9)
        self._call("global_order", _ptr(polar), _ptr(nem))
        return polar, nem.reshape(3, 3)


# ---- inputs without the CUDA library -----------------------------------------

INSERTION = {"random": 0, "random_nematic": 1, "random_polar": 2}


def oracle_n_bonds(params):
    """Bond count of a filament by the oracle's restatement of the
    reference's rule (src/filament.cpp:142-147)."""
    lib = ctypes.CDLL(ORACLE_SO)
    lib.sco_filament_n_bonds.restype = ctypes.c_int
    return lib.sco_filament_n_bonds(ctypes.byref(FilamentDesc(**params)))


def oracle_insert(n_dim, system_radius, seed, n_bonds, lengths, persistence_lengths,
                  diameter=1.0, max_attempts=10000, insertion="random"):
    """The oracle's random insertion with overlap rejection; same arguments
    and result as simcore_b200.insert_filaments (and the same configuration
    for the same seed)."""
    lib = ctypes.CDLL(ORACLE_SO)
    lib.sco_insert_filaments.restype = ctypes.c_int
    n_bonds = np.ascontiguousarray(n_bonds, dtype=np.int32)
    lengths = np.ascontiguousarray(lengths, dtype=np.float64)
    lps = np.ascontiguousarray(persistence_lengths, dtype=np.float64)
    xyz = np.zeros((int(np.sum(n_bonds + 1)), 3))
    rc = lib.sco_insert_filaments(ctypes.c_int(n_dim), ctypes.c_double(system_radius),
                                  ctypes.c_uint64(seed), ctypes.c_int(len(n_bonds)),
                                  _ptr(n_bonds), _ptr(lengths), _ptr(lps),
                                  ctypes.c_double(diameter),
                                  ctypes.c_int(INSERTION[insertion]),
                                  ctypes.c_int(max_attempts), _ptr(xyz))
    if rc != 0:
        raise RuntimeError("oracle insertion failed (%d)" % rc)
    return xyz


def workloads_module():
    """simcore_b200/workloads.py loaded on its own (numpy only), without the
    package and so without the CUDA library."""
    import importlib.util
    path = os.path.join(ROOT, "simcore_b200", "workloads.py")
    spec = importlib.util.spec_from_file_location("sc_workload_defs", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def oracle_workload(name, seed=0, scale=1.0):
    """(system, filaments, sites, replicas, crosslinks) of a bench workload,
    made by the oracle's insertion and bond-count rule: the configuration
    the library's own insertion makes, without loading the library."""
    wl = workloads_module()
    if name in wl.REPLICAS:
        system, fils, sites, reps = wl.make_replicas(name, seed=seed, insert=oracle_insert)
        return system, fils, sites, reps, None
    system, fils, sites = wl.make(name, scale, seed=seed, insert=oracle_insert)
    xl = wl.crosslinks(name, sites, fils, 2 * system["system_radius"], scale=scale, seed=seed,
                       n_bonds=oracle_n_bonds)
    return system, fils, sites, None, xl
