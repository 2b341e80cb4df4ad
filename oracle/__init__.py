"""oracle -- TEST INFRASTRUCTURE: Python access to the CPU oracle and to the
reference compiled from its own sources (oracle/_ref/, built by
oracle/build.py).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package.  The shipped library (irbc-code_b200/) never does.
"""
import contextlib
import ctypes as C
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DATA_DIR = os.path.join(os.path.dirname(HERE), "tests", "golden", "troph600")

D = C.POINTER(C.c_double)
I = C.POINTER(C.c_int32)


class Params(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("a", "Lx", "Ly", "Lz")] + [("Ns", C.c_int64)] + \
        [(n, C.c_double) for n in ("dtcd", "navg", "Theta", "walls", "mass", "cosalpha", "sinalpha")] + \
        [("Nt", C.c_int32)] + \
        [(n, C.c_double) for n in ("kappasa", "kappad", "kappav", "kappab", "pmass", "dtmd", "ks",
                                   "dthr", "FD", "Fg", "el0", "PRmass", "paraR", "Pi", "elap", "shear",
                                   "onrate", "offrate")] + \
        [("warm_steps", C.c_int64), ("warm_speed", C.c_double), ("out_every", C.c_int64),
         ("randno", C.c_int32), ("pad_", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad_"}


class Mesh(C.Structure):
    _fields_ = [("nv", C.c_int32), ("ne", C.c_int32), ("nt", C.c_int32), ("pad_", C.c_int32),
                ("e1", I), ("e2", I), ("l0", D), ("kappap", D), ("es1", I), ("es2", I), ("iedge", I),
                ("t1", I), ("t2", I), ("t3", I), ("cmx", D), ("cmy", D), ("cmz", D), ("tarea", D),
                ("Sarea0", C.c_double), ("Volume0", C.c_double), ("theta0", C.c_double),
                ("center", C.c_double * 3)]


class View(C.Structure):
    _fields_ = [("ns", C.c_int64)] + [(n, D) for n in ("sx", "sy", "sz", "svx", "svy", "svz")] + \
        [("spid", I), ("sindio", I), ("nv", C.c_int32), ("pad0_", C.c_int32)] + \
        [(n, D) for n in ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "poff", "pon")] + \
        [(n, I) for n in ("pid", "ix", "iy", "bondi", "bondl", "knob")] + \
        [(n, C.c_double * 3) for n in ("para", "paraV", "paraft", "parafdt")] + \
        [("paradx", C.c_int32), ("parady", C.c_int32), ("paraid", C.c_int32), ("nlig", C.c_int32),
         ("ligi", I), ("ncell", C.c_int64), ("llen", I), ("lcap", C.c_int64), ("lidx", I),
         ("Sarea", C.c_double), ("Volume", C.c_double), ("wallspeed", C.c_double),
         ("step", C.c_int64), ("colsteps", C.c_int32), ("upd", C.c_int32), ("filecc", C.c_int32),
         ("filec", C.c_int32)]


SOLVENT_D = ("sx", "sy", "sz", "svx", "svy", "svz")
SOLVENT_I = ("spid", "sindio")
VERT_D = ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "poff", "pon")
VERT_I = ("pid", "ix", "iy", "bondi", "bondl", "knob")
PARA_V = ("para", "paraV", "paraft", "parafdt")
PARA_I = ("paradx", "parady", "paraid")
SCALARS = ("Sarea", "Volume", "wallspeed")
COUNTERS = ("step", "colsteps", "upd", "filecc", "filec")


def _ptr(a, t):
    return a.ctypes.data_as(t)


class State:
    """Full dynamic state as numpy arrays (field names as in the C view)."""

    def __init__(self, ns, nv, nlig, ncell, lcap=0):
        self.a = {}
        for k in SOLVENT_D:
            self.a[k] = np.zeros(ns, np.float64)
        for k in SOLVENT_I:
            self.a[k] = np.zeros(ns, np.int32)
        for k in VERT_D:
            self.a[k] = np.zeros(nv, np.float64)
        for k in VERT_I:
            self.a[k] = np.zeros(nv, np.int32)
        self.a["ligi"] = np.zeros(nlig, np.int32)
        self.a["llen"] = np.zeros(ncell, np.int32)
        self.a["lidx"] = np.zeros(max(lcap, 1), np.int32)
        self.s = {k: np.zeros(3) for k in PARA_V}
        self.s.update({k: 0 for k in PARA_I + COUNTERS})
        self.s.update({k: 0.0 for k in SCALARS})
        self.ns, self.nv, self.nlig, self.ncell = ns, nv, nlig, ncell

    def view(self):
        v = View()
        v.ns, v.nv, v.nlig, v.ncell = self.ns, self.nv, self.nlig, self.ncell
        for k in SOLVENT_D + VERT_D:
            setattr(v, k, _ptr(self.a[k], D))
        for k in SOLVENT_I + VERT_I + ("ligi", "llen", "lidx"):
            setattr(v, k, _ptr(self.a[k], I))
        v.lcap = self.a["lidx"].size
        for k in PARA_V:
            getattr(v, k)[:] = [float(x) for x in self.s[k]]
        for k in PARA_I + COUNTERS + SCALARS:
            setattr(v, k, self.s[k])
        return v

    def absorb(self, v):
        for k in PARA_V:
            self.s[k] = np.array(getattr(v, k)[:])
        for k in PARA_I + COUNTERS + SCALARS:
            self.s[k] = getattr(v, k)

    def llists(self):
        off = np.concatenate([[0], np.cumsum(self.a["llen"], dtype=np.int64)])
        return off, self.a["lidx"][: off[-1]]

    def copy(self):
        o = State.__new__(State)
        o.a = {k: v.copy() for k, v in self.a.items()}
        o.s = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self.s.items()}
        o.ns, o.nv, o.nlig, o.ncell = self.ns, self.nv, self.nlig, self.ncell
        return o


class MeshArrays:
    def __init__(self, nv, ne, nt):
        self.nv, self.ne, self.nt = nv, ne, nt
        self.a = {k: np.zeros(ne, np.int32) for k in ("e1", "e2", "es1", "es2", "iedge")}
        self.a.update({k: np.zeros(ne) for k in ("l0", "kappap")})
        self.a.update({k: np.zeros(nt, np.int32) for k in ("t1", "t2", "t3")})
        self.a.update({k: np.zeros(nt) for k in ("cmx", "cmy", "cmz", "tarea")})
        self.s = {"Sarea0": 0.0, "Volume0": 0.0, "theta0": 0.0, "center": np.zeros(3)}

    def struct(self):
        m = Mesh()
        m.nv, m.ne, m.nt = self.nv, self.ne, self.nt
        for k, arr in self.a.items():
            setattr(m, k, _ptr(arr, I if arr.dtype == np.int32 else D))
        m.Sarea0, m.Volume0, m.theta0 = self.s["Sarea0"], self.s["Volume0"], self.s["theta0"]
        m.center[:] = [float(x) for x in self.s["center"]]
        return m

    def absorb(self, m):
        self.s.update(Sarea0=m.Sarea0, Volume0=m.Volume0, theta0=m.theta0, center=np.array(m.center[:]))


def load_mesh_files(vfile, efile, tfile):
    """Reads the reference's mesh files (maincode.cpp:174-272): V as
    'x y z' lines, E and T 1-based index lines.  Returns V, 0-based E, T."""
    V = np.loadtxt(vfile, dtype=np.float64).reshape(-1, 3)
    E = np.loadtxt(efile, dtype=np.int64).reshape(-1, 2) - 1
    T = np.loadtxt(tfile, dtype=np.int64).reshape(-1, 3) - 1
    return V, E.astype(np.int32), T.astype(np.int32)


def troph_files():
    """The shipped 600-vertex trophozoite mesh: the byte-identical copy kept
    as a test fixture in tests/golden/troph600 (test_oracle_vs_ref.py checks
    it against the reference's own files where the reference tree is)."""
    names = ("TrophV600.dat", "TrophE600.dat", "TrophT600.dat")
    if all(os.path.exists(os.path.join(DATA_DIR, n)) for n in names):
        return tuple(os.path.join(DATA_DIR, n) for n in names)
    raise FileNotFoundError("trophozoite mesh files not found in " + DATA_DIR)


# ------------------------------------------------------------------- oracle
_orc = None


def liboracle():
    global _orc
    if _orc is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            from . import build
            build.build_oracle()
        L = C.CDLL(path)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(Params), C.c_uint64]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_init.argtypes = [C.c_void_p, D, C.c_int32, I, C.c_int32, I, C.c_int32, C.c_int32, C.c_int32]
        L.orc_init_report.argtypes = [C.c_void_p, D]
        for f in ("orc_set_state", "orc_get_state"):
            getattr(L, f).argtypes = [C.c_void_p, C.POINTER(View)]
        for f in ("orc_set_mesh", "orc_get_mesh"):
            getattr(L, f).argtypes = [C.c_void_p, C.POINTER(Mesh)]
        L.orc_llist_total.restype = C.c_int64
        L.orc_llist_total.argtypes = [C.c_void_p]
        L.orc_ncell.restype = C.c_int64
        L.orc_ncell.argtypes = [C.c_void_p]
        for f in ("orc_last_normals", "orc_last_bond_draws"):
            getattr(L, f).restype = C.c_uint64
            getattr(L, f).argtypes = [C.c_void_p]
        for f in ("orc_collide", "orc_bond_dynamics", "orc_step"):
            getattr(L, f).argtypes = [C.c_void_p, C.c_int64]
        for f in ("orc_llist_update", "orc_stream", "orc_total_va", "orc_pfdt", "orc_forces",
                  "orc_step_part1", "orc_step_part2"):
            getattr(L, f).argtypes = [C.c_void_p]
        L.orc_reflection.restype = C.c_double
        L.orc_reflection.argtypes = [C.c_void_p, C.c_int64]
        L.orc_solve_cubic.restype = C.c_double
        L.orc_solve_cubic.argtypes = [C.c_double] * 3
        L.orc_solve_p3.restype = C.c_int
        L.orc_solve_p3.argtypes = [D, C.c_double, C.c_double, C.c_double]
        L.orc_params_default.argtypes = [C.POINTER(Params)]
        L.orc_write_rbcdata.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
        L.orc_write_stl.argtypes = [C.c_void_p, C.c_char_p]
        _orc = L
    return _orc


def default_params(**over):
    p = Params()
    liboracle().orc_params_default(C.byref(p))
    for k, v in over.items():
        setattr(p, k, v)
    return p


class Oracle:
    """One simulation held by the CPU oracle."""

    def __init__(self, params, seed):
        self.L = liboracle()
        self.p = params
        self.seed = seed
        self.h = self.L.orc_create(C.byref(params), seed)
        self.ncell = self.L.orc_ncell(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def init(self, V, E, T, nknobs, sort=True):
        V = np.ascontiguousarray(V, np.float64)
        E = np.ascontiguousarray(E, np.int32)
        T = np.ascontiguousarray(T, np.int32)
        r = self.L.orc_init(self.h, _ptr(V, D), len(V), _ptr(E, I), len(E), _ptr(T, I), len(T),
                            nknobs, 1 if sort else 0)
        assert r == 0
        self.nv, self.ne, self.nt = len(V), len(E), len(T)

    def report(self):
        out = np.zeros(9)
        self.L.orc_init_report(self.h, _ptr(out, D))
        return out

    def get_mesh(self):
        m0 = Mesh()
        self.L.orc_get_mesh(self.h, C.byref(m0))
        M = MeshArrays(m0.nv, m0.ne, m0.nt)
        m = M.struct()
        self.L.orc_get_mesh(self.h, C.byref(m))
        M.absorb(m)
        return M

    def set_mesh(self, M):
        self._mesh_keep = M
        m = M.struct()
        self.L.orc_set_mesh(self.h, C.byref(m))

    def get_state(self):
        v0 = View()
        self.L.orc_get_state(self.h, C.byref(v0))
        st = State(v0.ns, v0.nv, v0.nlig, v0.ncell, int(self.L.orc_llist_total(self.h)))
        v = st.view()
        assert self.L.orc_get_state(self.h, C.byref(v)) == 0
        st.absorb(v)
        return st

    def set_state(self, st):
        v = st.view()
        assert self.L.orc_set_state(self.h, C.byref(v)) == 0

    def __getattr__(self, name):
        f = getattr(self.L, "orc_" + name)
        return lambda *a: f(self.h, *a)


# --------------------------------------------------------------- reference
_refs = {}
REF_CB = C.CFUNCTYPE(None, C.c_int64)


def ref_lib_path(variant):
    return os.path.join(HERE, "_ref", variant, "libref.so")


def libref(variant):
    if variant not in _refs:
        path = ref_lib_path(variant)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = C.CDLL(path)
        L.ref_run.restype = C.c_int
        L.ref_run.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.c_int64, REF_CB, C.c_uint64, C.c_int]
        L.ref_get_params.argtypes = [C.POINTER(Params)]
        L.ref_get_mesh.argtypes = [C.POINTER(Mesh)]
        L.ref_get_state.argtypes = [C.POINTER(View), C.c_int64]
        L.ref_set_state.argtypes = [C.POINTER(View)]
        L.ref_llist_total.restype = C.c_int64
        L.ref_step_times.restype = C.c_int64
        L.ref_step_times.argtypes = [D, C.c_int64]
        for f in ("ref_call_collide", "ref_call_bond_dynamics"):
            getattr(L, f).argtypes = [C.c_uint64]
        L.ref_call_reflection.restype = C.c_double
        L.ref_call_reflection.argtypes = [C.c_int]
        L.ref_call_solve.restype = C.c_double
        L.ref_call_solve.argtypes = [C.c_double] * 3
        L.ref_call_solvep3.restype = C.c_int
        L.ref_call_solvep3.argtypes = [D, C.c_double, C.c_double, C.c_double]
        L.ref_uniform_cursor.restype = C.c_uint64
        L.ref_normal_cursor.restype = C.c_uint64
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_call_filewrite.argtypes = [C.c_char_p]
        _refs[variant] = L
    return _refs[variant]


@contextlib.contextmanager
def _in_dir(d):
    old = os.getcwd()
    os.chdir(d)
    try:
        yield
    finally:
        os.chdir(old)


class Reference:
    """The reference's own main() run under the hooks of oracle/ref_hooks.cpp."""

    def __init__(self, variant="small", threads=1):
        self.variant = variant
        self.L = libref(variant)
        self.L.ref_set_threads(threads)
        p = Params()
        self.L.ref_get_params(C.byref(p))
        self.p = p

    def run(self, vfile, efile, tfile, nknobs, stop_step, seed, onrate=0.005, offrate=0.015,
            on_step=None, fast_init=0, workdir=None, stl=0):
        """Runs main() until the TotalVA snapshot of step `stop_step`.
        on_step(step) is called at each step's TotalVA point; stl is main()'s
        stl_flag argument (1: an rbc<k>.stl beside each RBCdata record)."""
        def cb(s):
            if on_step is not None:
                on_step(int(s))
        self._cb = REF_CB(cb)
        wd = workdir or tempfile.mkdtemp(prefix="irbc_ref_")
        args = ["MAIN", repr(onrate), repr(offrate), os.path.abspath(vfile), os.path.abspath(efile),
                os.path.abspath(tfile), str(nknobs), os.path.join(wd, "RBCdata.dat"), str(int(stl))]
        argv = (C.c_char_p * len(args))(*[a.encode() for a in args])
        self.p.onrate, self.p.offrate = onrate, offrate
        with _in_dir(wd):
            r = self.L.ref_run(len(args), argv, stop_step, self._cb, seed, fast_init)
        self.workdir = wd
        return r

    def get_mesh(self):
        m0 = Mesh()
        self.L.ref_get_mesh(C.byref(m0))
        M = MeshArrays(m0.nv, m0.ne, m0.nt)
        m = M.struct()
        self.L.ref_get_mesh(C.byref(m))
        M.absorb(m)
        return M

    def get_state(self, step):
        v0 = View()
        self.L.ref_get_state(C.byref(v0), step)
        st = State(v0.ns, v0.nv, v0.nlig, v0.ncell, int(self.L.ref_llist_total()))
        v = st.view()
        assert self.L.ref_get_state(C.byref(v), step) == 0
        st.absorb(v)
        return st

    def set_state(self, st):
        v = st.view()
        assert self.L.ref_set_state(C.byref(v)) == 0

    def step_times(self):
        out = np.zeros(1 << 16)
        n = self.L.ref_step_times(_ptr(out, D), out.size)
        return out[:n].copy()

    def __getattr__(self, name):
        return getattr(self.L, "ref_" + name)


def params_of_reference(variant):
    return Reference(variant).p


def compare_states(a, b, fields=None, exact=True, rtol=0.0):
    """Returns {field: max abs diff} (or mismatch count for ints)."""
    out = {}
    for k in fields or a.a.keys():
        x, y = a.a[k], b.a[k]
        if k == "lidx":
            ox, lx = a.llists()
            oy, ly = b.llists()
            out[k] = int((lx != ly).sum()) if lx.shape == ly.shape else -1
            continue
        if x.shape != y.shape:
            out[k] = -1
            continue
        if x.dtype.kind == "f":
            out[k] = float(np.max(np.abs(x - y))) if x.size else 0.0
        else:
            out[k] = int((x != y).sum())
    return out
