"""irbc_b200 -- Python access to libirbc.so (the B200 iRBC timestep).

A thin ctypes layer over the C ABI of include/irbc.h, used by the tests,
bench.py and the MAIN driver.  All arithmetic runs in the CUDA library; if
libirbc.so is missing or cannot reach a GPU the calls raise, there is no
fallback.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "libirbc.so")
HEADER = os.path.join(ROOT, "include", "irbc.h")

FP64, FP32 = 0, 1
D = C.POINTER(C.c_double)
I = C.POINTER(C.c_int32)


class Result(C.Structure):
    """irbc_result"""
    _fields_ = [("id", C.c_int64), ("status", C.c_int32), ("pad_", C.c_int32), ("steps", C.c_int64),
                ("ns", C.c_int64), ("t_submit", C.c_double), ("t_start", C.c_double), ("t_end", C.c_double),
                ("obs", C.c_double * 8), ("handle", C.c_void_p)]


class IrbcError(RuntimeError):
    pass


class Params(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("a", "Lx", "Ly", "Lz")] + [("Ns", C.c_int64)] + \
        [(n, C.c_double) for n in ("dtcd", "navg", "Theta", "walls", "mass", "cosalpha", "sinalpha")] + \
        [("Nt", C.c_int32)] + \
        [(n, C.c_double) for n in ("kappasa", "kappad", "kappav", "kappab", "pmass", "dtmd", "ks",
                                   "dthr", "FD", "Fg", "el0", "PRmass", "paraR", "Pi", "elap", "shear",
                                   "onrate", "offrate")] + \
        [("warm_steps", C.c_int64), ("warm_speed", C.c_double), ("out_every", C.c_int64),
         ("randno", C.c_int32), ("pad_", C.c_int32), ("seed", C.c_uint64), ("precision", C.c_int32),
         ("device", C.c_int32)]


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


class Schedule(C.Structure):
    """irbc_schedule: how a batch launches its members' steps."""
    _fields_ = [("streams", C.c_int32), ("membrane", C.c_int32), ("graphs", C.c_int32), ("chunk", C.c_int32),
                ("fused", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# int (*)(int32_t candidate, void* ctx, double* seconds)
TUNE_MEASURE = C.CFUNCTYPE(C.c_int, C.c_int32, C.c_void_p, C.POINTER(C.c_double))
ERR_ARG, ERR_CAPACITY, ERR_HEALTH = -1, -4, -6
# bits of the health word (irbc_health)
HEALTH_SOLVENT, HEALTH_MEMBRANE = 1, 2


def tune_select(n, measure, repeats=3, margin=0.02):
    """irbc_tune_select over n candidates.  measure(i) runs candidate i once
    and returns its time in seconds, or None when it cannot run (skipped).
    Returns (best index, medians with -1 for skipped candidates)."""
    raised = []

    def cb(i, _ctx, out):
        if raised:
            return ERR_ARG
        try:
            t = measure(i)
        except Exception as e:  # an exception cannot cross the C frame
            raised.append(e)
            return ERR_ARG
        if t is None:
            return ERR_CAPACITY
        out[0] = float(t)
        return 0

    fn = TUNE_MEASURE(cb)
    med = (C.c_double * n)()
    best = C.c_int32(-1)
    rc = lib().irbc_tune_select(n, fn, None, repeats, margin, med, C.byref(best))
    if raised:
        raise raised[0]
    if rc != 0:
        raise IrbcError("irbc_tune_select failed (%d)" % rc)
    return best.value, list(med)


def exported_names():
    """Function names declared in include/irbc.h."""
    import re
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(irbc_[a-z0-9_]+)\s*\(", txt)))


_lib = None


def lib():
    """Loads libirbc.so (built by irbc-code_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise IrbcError("libirbc.so not built: run irbc-code_b200/build.py")
    L = C.CDLL(LIB_PATH)
    H = C.c_void_p
    L.irbc_params_default.argtypes = [C.POINTER(Params)]
    L.irbc_create.argtypes = [C.POINTER(Params), C.POINTER(H)]
    L.irbc_destroy.argtypes = [H]
    L.irbc_last_error.restype = C.c_char_p
    L.irbc_last_error.argtypes = [H]
    L.irbc_footprint_bytes.restype = C.c_int64
    L.irbc_footprint_bytes.argtypes = [C.POINTER(Params), C.c_int32, C.c_int32, C.c_int32]
    L.irbc_init.argtypes = [H, D, C.c_int32, I, C.c_int32, I, C.c_int32, C.c_int32]
    L.irbc_init_report.argtypes = [H, D]
    L.irbc_set_mesh.argtypes = [H, C.POINTER(Mesh)]
    L.irbc_get_mesh.argtypes = [H, C.POINTER(Mesh)]
    L.irbc_set_state.argtypes = [H, C.POINTER(View)]
    L.irbc_get_state.argtypes = [H, C.POINTER(View)]
    L.irbc_llist_total.restype = C.c_int64
    L.irbc_llist_total.argtypes = [H]
    L.irbc_ncell.restype = C.c_int64
    L.irbc_ncell.argtypes = [H]
    L.irbc_nlig.argtypes = [H]
    for f in ("irbc_step", "irbc_collide", "irbc_bond_dynamics"):
        getattr(L, f).argtypes = [H, C.c_int64]
    for f in ("irbc_step_part1", "irbc_step_part2", "irbc_llist_update", "irbc_stream", "irbc_total_va",
              "irbc_pfdt", "irbc_forces", "irbc_sync"):
        getattr(L, f).argtypes = [H]
    L.irbc_write_rbcdata.argtypes = [H, C.c_char_p, C.c_int32]
    L.irbc_write_stl.argtypes = [H, C.c_char_p]
    L.irbc_observables.argtypes = [H, D, C.c_int32]
    L.irbc_health.argtypes = [H, I]
    L.irbc_velocity_profile.argtypes = [H, D, C.c_int32]
    L.irbc_launch_count.restype = C.c_int64
    L.irbc_launch_count.argtypes = [H]
    L.irbc_profile_begin.argtypes = [H]
    L.irbc_set_graphs.argtypes = [H, C.c_int32]
    L.irbc_set_streams.argtypes = [H, C.c_int32]
    L.irbc_timer_begin.argtypes = [H]
    L.irbc_timer_end.argtypes = [H, D]
    L.irbc_record_bytes.restype = C.c_int64
    L.irbc_record_bytes.argtypes = [H]
    L.irbc_record_async.argtypes = [H, C.c_void_p, C.c_int64]
    L.irbc_set_membrane_kernels.argtypes = [H, C.c_int32]
    L.irbc_profile_end.argtypes = [H, D, C.c_int32]
    L.irbc_host_alloc.restype = C.c_void_p
    L.irbc_host_alloc.argtypes = [C.c_size_t]
    L.irbc_host_free.argtypes = [C.c_void_p]
    L.irbc_bin_particles.argtypes = [C.POINTER(Params), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                     C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
    L.irbc_bin_particles_noalloc.argtypes = L.irbc_bin_particles.argtypes
    B = C.c_void_p
    L.irbc_batch_create.argtypes = [C.c_int32, C.POINTER(B)]
    L.irbc_batch_destroy.argtypes = [B]
    L.irbc_batch_destroy.restype = None
    L.irbc_batch_add.argtypes = [B, H]
    L.irbc_batch_remove.argtypes = [B, H]
    L.irbc_batch_size.argtypes = [B]
    L.irbc_batch_step.argtypes = [B, C.c_int64]
    L.irbc_batch_set_schedule.argtypes = [B, C.POINTER(Schedule)]
    L.irbc_batch_get_schedule.argtypes = [B, C.POINTER(Schedule)]
    L.irbc_tune_select.argtypes = [C.c_int32, TUNE_MEASURE, C.c_void_p, C.c_int32, C.c_double, D, I]
    L.irbc_batch_autotune.argtypes = [B, C.c_int64, C.c_int32, C.c_double, C.POINTER(Schedule),
                                      C.POINTER(C.c_int64)]
    L.irbc_server_create.argtypes = [C.c_int32, C.c_int64, C.c_int32, C.c_int64, C.POINTER(B)]
    L.irbc_server_submit.argtypes = [B, C.POINTER(Params), D, C.c_int32, I, C.c_int32, I, C.c_int32, C.c_int32,
                                     C.c_int64, C.c_int32, C.POINTER(C.c_int64)]
    L.irbc_server_poll.argtypes = [B, C.POINTER(Result), C.c_int32, C.c_double]
    L.irbc_server_status.argtypes = [B, C.POINTER(C.c_int64)]
    L.irbc_server_clock.restype = C.c_double
    L.irbc_server_clock.argtypes = [B]
    L.irbc_server_set_schedule.argtypes = [B, C.POINTER(Schedule)]
    L.irbc_server_release.argtypes = [B, H]
    L.irbc_server_destroy.argtypes = [B]
    L.irbc_server_destroy.restype = None
    _lib = L
    return L


def default_params(**over):
    p = Params()
    lib().irbc_params_default(C.byref(p))
    for k, v in over.items():
        setattr(p, k, v)
    return p


def _p(a, t):
    return a.ctypes.data_as(t)


class State:
    """Host copy of a simulation state in the reference's layout."""
    SOLVENT_D = ("sx", "sy", "sz", "svx", "svy", "svz")
    SOLVENT_I = ("spid", "sindio")
    VERT_D = ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "poff", "pon")
    VERT_I = ("pid", "ix", "iy", "bondi", "bondl", "knob")
    PARA_V = ("para", "paraV", "paraft", "parafdt")
    SCAL = ("paradx", "parady", "paraid", "Sarea", "Volume", "wallspeed", "step", "colsteps", "upd",
            "filecc", "filec")

    def __init__(self, ns, nv, nlig, ncell, lcap=1, solvent=True, llist=True):
        self.ns, self.nv, self.nlig, self.ncell = ns, nv, nlig, ncell
        self.a = {}
        if solvent:
            self.a.update({k: np.zeros(ns) for k in self.SOLVENT_D})
            self.a.update({k: np.zeros(ns, np.int32) for k in self.SOLVENT_I})
        self.a.update({k: np.zeros(nv) for k in self.VERT_D})
        self.a.update({k: np.zeros(nv, np.int32) for k in self.VERT_I})
        self.a["ligi"] = np.zeros(nlig, np.int32)
        if llist:
            self.a["llen"] = np.zeros(ncell, np.int32)
            self.a["lidx"] = np.zeros(max(lcap, 1), np.int32)
        self.s = {k: np.zeros(3) for k in self.PARA_V}
        self.s.update({k: 0 for k in self.SCAL})

    def view(self):
        v = View()
        v.ns, v.nv, v.nlig, v.ncell = self.ns, self.nv, self.nlig, self.ncell
        for k, arr in self.a.items():
            setattr(v, k, _p(arr, D if arr.dtype == np.float64 else I))
        if "lidx" in self.a:
            v.lcap = self.a["lidx"].size
        for k in self.PARA_V:
            getattr(v, k)[:] = [float(x) for x in self.s[k]]
        for k in self.SCAL:
            setattr(v, k, self.s[k])
        return v

    def absorb(self, v):
        for k in self.PARA_V:
            self.s[k] = np.array(getattr(v, k)[:])
        for k in self.SCAL:
            self.s[k] = getattr(v, k)

    def copy(self):
        return State.from_other(self)

    @classmethod
    def from_other(cls, other):
        """Copies any object with .a/.s dicts and ns/nv/nlig/ncell (e.g. an oracle state)."""
        st = cls.__new__(cls)
        st.ns, st.nv, st.nlig, st.ncell = other.ns, other.nv, other.nlig, other.ncell
        st.a = {k: np.ascontiguousarray(v).copy() for k, v in other.a.items()}
        st.s = {k: (np.array(v).copy() if isinstance(v, np.ndarray) else v) for k, v in other.s.items()}
        return st


class Simulation:
    """One simulation on one GPU (a handle of libirbc.so)."""

    def __init__(self, params):
        self.L = lib()
        self.params = params
        self.h = C.c_void_p()
        rc = self.L.irbc_create(C.byref(params), C.byref(self.h))
        if rc != 0:
            why = self.L.irbc_last_error(None)
            raise IrbcError("irbc_create failed (%d): %s" % (rc, why.decode() if why else "bad parameters"))
        self.ncell = int(self.L.irbc_ncell(self.h))
        self.nlig = int(self.L.irbc_nlig(self.h))
        self.nv = 0

    @classmethod
    def adopt(cls, handle, params, nv, server=None):
        """wraps a handle the library created (a server result with keep = 1);
        close() hands it back to `server` (irbc_server_release) while that
        server is open"""
        sim = cls.__new__(cls)
        sim.L = lib()
        sim._server = server
        sim.params = params
        sim.h = C.c_void_p(handle)
        sim.ncell = int(sim.L.irbc_ncell(sim.h))
        sim.nlig = int(sim.L.irbc_nlig(sim.h))
        sim.nv = nv
        return sim

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            srv = getattr(self, "_server", None)
            if srv is not None and srv.s.value:
                if self.L.irbc_server_release(srv.s, self.h) != 0:
                    self.L.irbc_destroy(self.h)
            else:
                self.L.irbc_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc, what):
        if rc != 0:
            raise IrbcError("%s failed (%d): %s" % (what, rc, self.L.irbc_last_error(self.h).decode()))

    def init(self, V, E, T, nknobs):
        V = np.ascontiguousarray(V, np.float64)
        E = np.ascontiguousarray(E, np.int32)
        T = np.ascontiguousarray(T, np.int32)
        self._ck(self.L.irbc_init(self.h, _p(V, D), len(V), _p(E, I), len(E), _p(T, I), len(T), nknobs),
                 "irbc_init")
        self.nv = len(V)

    def report(self):
        out = np.zeros(9)
        self._ck(self.L.irbc_init_report(self.h, _p(out, D)), "irbc_init_report")
        return out

    def set_mesh(self, M):
        """M: object with .a dict (e1,e2,l0,kappap,es1,es2,iedge,t1,t2,t3,tarea,...) and .s scalars."""
        m = Mesh()
        m.nv, m.ne, m.nt = M.nv, M.ne, M.nt
        keep = {}
        for k in ("e1", "e2", "es1", "es2", "iedge", "t1", "t2", "t3"):
            keep[k] = np.ascontiguousarray(M.a[k], np.int32)
            setattr(m, k, _p(keep[k], I))
        for k in ("l0", "kappap", "tarea", "cmx", "cmy", "cmz"):
            keep[k] = np.ascontiguousarray(M.a[k], np.float64)
            setattr(m, k, _p(keep[k], D))
        m.Sarea0, m.Volume0, m.theta0 = M.s["Sarea0"], M.s["Volume0"], M.s["theta0"]
        m.center[:] = [float(x) for x in M.s["center"]]
        self._ck(self.L.irbc_set_mesh(self.h, C.byref(m)), "irbc_set_mesh")
        self.nv = M.nv

    def get_mesh_arrays(self):
        m0 = Mesh()
        self._ck(self.L.irbc_get_mesh(self.h, C.byref(m0)), "irbc_get_mesh")
        a = {k: np.zeros(m0.ne, np.int32) for k in ("e1", "e2", "es1", "es2", "iedge")}
        a.update({k: np.zeros(m0.ne) for k in ("l0", "kappap")})
        a.update({k: np.zeros(m0.nt, np.int32) for k in ("t1", "t2", "t3")})
        a.update({k: np.zeros(m0.nt) for k in ("cmx", "cmy", "cmz", "tarea")})
        m = Mesh()
        m.nv, m.ne, m.nt = m0.nv, m0.ne, m0.nt
        for k, arr in a.items():
            setattr(m, k, _p(arr, I if arr.dtype == np.int32 else D))
        self._ck(self.L.irbc_get_mesh(self.h, C.byref(m)), "irbc_get_mesh")
        return a, {"Sarea0": m.Sarea0, "Volume0": m.Volume0, "theta0": m.theta0, "center": np.array(m.center[:])}

    def set_state(self, st):
        v = st.view()
        self._ck(self.L.irbc_set_state(self.h, C.byref(v)), "irbc_set_state")

    def get_state(self, solvent=True, llist=True):
        lcap = int(self.L.irbc_llist_total(self.h)) if llist else 1
        st = State(self.params.Ns, self.nv, self.nlig, self.ncell, lcap, solvent=solvent, llist=llist)
        v = st.view()
        self._ck(self.L.irbc_get_state(self.h, C.byref(v)), "irbc_get_state")
        st.absorb(v)
        return st

    def step(self, n=1):
        self._ck(self.L.irbc_step(self.h, n), "irbc_step")

    def sync(self):
        self._ck(self.L.irbc_sync(self.h), "irbc_sync")

    def health(self):
        """the health word after the queued work (0: healthy; HEALTH_SOLVENT,
        HEALTH_MEMBRANE bits)"""
        f = C.c_int32(0)
        self._ck(self.L.irbc_health(self.h, C.byref(f)), "irbc_health")
        return f.value

    def call(self, name, *args):
        self._ck(getattr(self.L, "irbc_" + name)(self.h, *args), "irbc_" + name)

    def observables(self):
        out = np.zeros(16)
        self._ck(self.L.irbc_observables(self.h, _p(out, D), 16), "irbc_observables")
        return out

    def velocity_profile(self, nbins):
        out = np.zeros(nbins)
        self._ck(self.L.irbc_velocity_profile(self.h, _p(out, D), nbins), "irbc_velocity_profile")
        return out

    def write_rbcdata(self, path, append=True):
        self._ck(self.L.irbc_write_rbcdata(self.h, path.encode(), 1 if append else 0), "irbc_write_rbcdata")

    def write_stl(self, path):
        self._ck(self.L.irbc_write_stl(self.h, path.encode()), "irbc_write_stl")

    def launch_count(self):
        return int(self.L.irbc_launch_count(self.h))

    def set_graphs(self, on):
        """captured 24-step CUDA graphs in step() (default off)"""
        self._ck(self.L.irbc_set_graphs(self.h, 1 if on else 0), "irbc_set_graphs")

    def record_async(self, pinned):
        """queue the RBCdata record (x, y, z, ix, iy, bondi of every vertex)
        into a PinnedArray of irbc_record_bytes bytes; valid after sync()"""
        self._ck(self.L.irbc_record_async(self.h, C.c_void_p(pinned.ptr), pinned.array.nbytes), "irbc_record_async")

    def record_bytes(self):
        return int(self.L.irbc_record_bytes(self.h))

    def timer_begin(self):
        self._ck(self.L.irbc_timer_begin(self.h), "irbc_timer_begin")

    def timer_end(self):
        """device ms since timer_begin (two events on the handle's stream)"""
        out = np.zeros(1)
        self._ck(self.L.irbc_timer_end(self.h, _p(out, D)), "irbc_timer_end")
        return float(out[0])

    def set_streams(self, n):
        """2 (default): membrane kernels on a second stream; 1: one stream"""
        self._ck(self.L.irbc_set_streams(self.h, int(n)), "irbc_set_streams")

    def set_membrane_kernels(self, mode):
        """1: wide kernels (default); 2: one block (meshes up to 1024 vertices)"""
        self._ck(self.L.irbc_set_membrane_kernels(self.h, int(mode)), "irbc_set_membrane_kernels")

    def profile_begin(self):
        self._ck(self.L.irbc_profile_begin(self.h), "irbc_profile_begin")

    def profile_end(self):
        """dict of CUDA-event times (ms) since profile_begin"""
        out = np.zeros(10)
        self._ck(self.L.irbc_profile_end(self.h, _p(out, D), 10), "irbc_profile_end")
        return dict(total_ms=out[0], stream_ms=out[1], stream_steps=int(out[2]), collide_ms=out[3],
                    collides=int(out[4]), membrane_ms=out[5], membrane_groups=int(out[6]),
                    launches=int(out[7]), bulk_ms=out[8], bulk_launches=int(out[9]))


class Batch:
    """Independent simulations stepped together (irbc_batch_*)."""

    def __init__(self, nthreads=4):
        self.L = lib()
        self.b = C.c_void_p()
        if self.L.irbc_batch_create(nthreads, C.byref(self.b)) != 0:
            raise IrbcError("irbc_batch_create failed")
        self.members = []

    def add(self, sim):
        if self.L.irbc_batch_add(self.b, sim.h) != 0:
            raise IrbcError("irbc_batch_add failed")
        self.members.append(sim)

    def remove(self, sim):
        if self.L.irbc_batch_remove(self.b, sim.h) != 0:
            raise IrbcError("irbc_batch_remove failed")
        self.members.remove(sim)

    def step(self, n):
        rc = self.L.irbc_batch_step(self.b, n)
        if rc != 0:
            raise IrbcError("irbc_batch_step failed (%d)" % rc)

    def schedule(self):
        s = Schedule()
        if self.L.irbc_batch_get_schedule(self.b, C.byref(s)) != 0:
            raise IrbcError("irbc_batch_get_schedule failed")
        return s.as_dict()

    def set_schedule(self, **fields):
        s = Schedule(**{**self.schedule(), **fields})
        rc = self.L.irbc_batch_set_schedule(self.b, C.byref(s))
        if rc != 0:
            raise IrbcError("irbc_batch_set_schedule failed (%d)" % rc)

    def autotune(self, trial_steps=120, repeats=3, margin=0.02):
        """Tunes the launch schedule on the members themselves; returns
        (schedule dict, steps every member advanced while tuning)."""
        s = Schedule()
        taken = C.c_int64(0)
        rc = self.L.irbc_batch_autotune(self.b, trial_steps, repeats, margin, C.byref(s), C.byref(taken))
        if rc != 0:
            raise IrbcError("irbc_batch_autotune failed (%d)" % rc)
        return s.as_dict(), taken.value

    def close(self):
        if self.b.value:
            self.L.irbc_batch_destroy(self.b)
            self.b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Request loop over whole simulations (irbc_server_*): admission by
    device-memory footprint, rounds of round_steps steps, results as they
    finish."""

    def __init__(self, device=0, budget_bytes=0, nthreads=4, round_steps=240):
        self.L = lib()
        self.s = C.c_void_p()
        rc = self.L.irbc_server_create(device, budget_bytes, nthreads, round_steps, C.byref(self.s))
        if rc != 0:
            raise IrbcError("irbc_server_create failed (%d)" % rc)
        self.params = {}

    def submit(self, params, V, E, T, nknobs, nsteps, keep=False):
        V = np.ascontiguousarray(V, np.float64)
        E = np.ascontiguousarray(E, np.int32)
        T = np.ascontiguousarray(T, np.int32)
        rid = C.c_int64()
        rc = self.L.irbc_server_submit(self.s, C.byref(params), _p(V, D), len(V), _p(E, I), len(E), _p(T, I),
                                       len(T), nknobs, nsteps, 1 if keep else 0, C.byref(rid))
        if rc != 0:
            raise IrbcError("irbc_server_submit failed (%d)" % rc)
        self.params[rid.value] = (params, len(V))
        return rid.value

    def poll(self, max_results=64, wait=0.0):
        buf = (Result * max_results)()
        n = self.L.irbc_server_poll(self.s, buf, max_results, wait)
        out = []
        for r in buf[:max(0, n)]:
            d = dict(id=r.id, status=r.status, steps=r.steps, ns=r.ns, t_submit=r.t_submit, t_start=r.t_start,
                     t_end=r.t_end, obs=np.array(r.obs[:]), sim=None)
            if r.handle:
                params, nv = self.params[r.id]
                d["sim"] = Simulation.adopt(r.handle, params, nv, server=self)
            out.append(d)
        return out

    def status(self):
        out = (C.c_int64 * 6)()
        self.L.irbc_server_status(self.s, out)
        return dict(pending=out[0], active=out[1], results=out[2], used=out[3], budget=out[4],
                    particle_steps=out[5])

    def set_schedule(self, streams=2, membrane=1, graphs=0, chunk=24, fused=1):
        """Launch schedule for simulations admitted from now on."""
        s = Schedule(streams, membrane, graphs, chunk, fused)
        rc = self.L.irbc_server_set_schedule(self.s, C.byref(s))
        if rc != 0:
            raise IrbcError("irbc_server_set_schedule failed (%d)" % rc)

    def clock(self):
        return float(self.L.irbc_server_clock(self.s))

    def close(self):
        if self.s.value:
            self.L.irbc_server_destroy(self.s)
            self.s = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PinnedArray:
    """numpy view of page-locked host memory from irbc_host_alloc."""

    def __init__(self, n, dtype):
        dtype = np.dtype(dtype)
        self.ptr = lib().irbc_host_alloc(max(1, n) * dtype.itemsize)
        if not self.ptr:
            raise IrbcError("irbc_host_alloc failed")
        buf = (C.c_char * (max(1, n) * dtype.itemsize)).from_address(self.ptr)
        self.array = np.frombuffer(buf, dtype=dtype, count=n)

    def __del__(self):
        try:
            if self.ptr:
                lib().irbc_host_free(self.ptr)
                self.ptr = None
        except Exception:
            pass
