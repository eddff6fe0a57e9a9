"""ctypes view of oracle/liboracle.so -- the CPU checker (test infrastructure).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this.
"""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(ROOT, "oracle", "liboracle.so")

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            import subprocess
            subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        sig = {
            "oracle_tree_sum": (ctypes.c_double, [_D, ctypes.c_long]),
            "oracle_fm": (ctypes.c_double, [ctypes.c_int, ctypes.c_double]),
            "oracle_dendrite_new": (vp, [ctypes.c_int] * 5 + [_D, ctypes.c_int]),
            "oracle_dendrite_init_cone": (None, [vp]),
            "oracle_dendrite_set": (None, [vp, _D, _D]),
            "oracle_dendrite_step": (None, [vp, ctypes.c_int, ctypes.c_int]),
            "oracle_dendrite_get": (None, [vp, _D, _D, _I, _I, _I, _I]),
            "oracle_dendrite_tip": (ctypes.c_double, [vp]),
            "oracle_dendrite_set_flags": (None, [vp, _I, _I]),
            "oracle_tip_profile": (None, [_D, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _I,
                                          ctypes.POINTER(ctypes.c_int)]),
            "oracle_size_distribution": (ctypes.c_long, [_D, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D,
                                                         ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_long),
                                                         ctypes.c_long]),
            "oracle_dendrite_free": (None, [vp]),
            "oracle_modelb_new": (vp, [ctypes.c_int] * 5 + [_D, ctypes.c_int, ctypes.c_int]),
            "oracle_modelb_init_uniform": (None, [vp, _D, _D, _D, ctypes.c_double, ctypes.c_double]),
            "oracle_modelb_init_mt": (None, [vp, ctypes.c_ulonglong, ctypes.c_double, ctypes.c_double]),
            "oracle_modelb_set": (None, [vp, _D, _D, _D]),
            "oracle_modelb_step": (None, [vp, ctypes.c_int, ctypes.c_int]),
            "oracle_modelb_get_field": (None, [vp, ctypes.c_int, _D]),
            "oracle_modelb_get_flags": (None, [vp, _I, _I]),
            "oracle_modelb_last_avg": (None, [vp, _D]),
            "oracle_modelb_free": (None, [vp]),
            "oracle_modelb_set_owned": (None, [vp, ctypes.c_int, ctypes.c_int]),
            "oracle_modelb_set_field": (None, [vp, ctypes.c_int, _D]),
            "oracle_modelb_set_flags": (None, [vp, _I]),
            "oracle_kh_new": (vp, [ctypes.c_int] * 4 + [_D, ctypes.c_int]),
            "oracle_kh_init_smooth": (None, [vp]),
            "oracle_kh_set_primitive": (None, [vp, _D, _D, _D, _D]),
            "oracle_kh_step": (None, [vp, ctypes.c_int, ctypes.c_int]),
            "oracle_kh_get_field": (None, [vp, ctypes.c_int, _D]),
            "oracle_kh_get_flags": (None, [vp, _I, _I]),
            "oracle_kh_free": (None, [vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def dptr(a):
    return a.ctypes.data_as(_D)


def iptr(a):
    return a.ctypes.data_as(_I)


# parameter vectors in the order the oracle expects (== Input.txt order)
DENDRITE_KEYS = ["dt", "dx", "delta", "tau", "epsilon", "alpha", "gamma", "Delta", "metric_p", "metric_T"]
MODELB_KEYS = ["dt", "dx", "chi_xy", "chi_xz", "chi_yz", "chi_xb", "chi_yb", "chi_zb", "vx", "vy", "vz",
               "rx", "ry", "rz", "n", "m", "eps_x", "eps_y", "eps_z", "eps_phi", "M_x", "M_y", "M_z", "M_phi",
               "x0", "y0", "z0", "K", "z_crit", "p_gel", "k_0", "metric_eps"]
KH_KEYS = ["dt", "dx", "dy", "metric_eps", "gamma"]


class OracleDendrite:
    def __init__(self, nx, ny, nz, edge, prm, bc=0, libm=False):
        self.n = nx * ny * nz
        self.shape = (nz, ny, nx)
        self.nb = ((nx - 1) // edge + 1) * ((ny - 1) // edge + 1) * (1 if nz == 1 else (nz - 1) // edge + 1)
        v = np.array([prm[k] for k in DENDRITE_KEYS], dtype=np.float64)
        self.h = lib().oracle_dendrite_new(nx, ny, nz, edge, bc, dptr(v), int(libm))

    def init_cone(self):
        lib().oracle_dendrite_init_cone(self.h)

    def set_fields(self, p, T):
        p = np.ascontiguousarray(p, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.float64)
        lib().oracle_dendrite_set(self.h, dptr(p), dptr(T))

    def set_flags(self, wake_p, wake_T):
        a = np.ascontiguousarray(wake_p, dtype=np.int32)
        b = np.ascontiguousarray(wake_T, dtype=np.int32)
        lib().oracle_dendrite_set_flags(self.h, iptr(a), iptr(b))

    def step(self, n=1, mode=1):
        lib().oracle_dendrite_step(self.h, n, mode)

    def get(self):
        p = np.empty(self.n); T = np.empty(self.n)
        wp = np.empty(self.nb, np.int32); wT = np.empty(self.nb, np.int32)
        np_ = np.empty(self.nb, np.int32); nT = np.empty(self.nb, np.int32)
        lib().oracle_dendrite_get(self.h, dptr(p), dptr(T), iptr(wp), iptr(wT), iptr(np_), iptr(nT))
        return dict(p=p.reshape(self.shape), T=T.reshape(self.shape), wake_p=wp, wake_T=wT, next_p=np_, next_T=nT)

    def tip(self):
        return lib().oracle_dendrite_tip(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_dendrite_free(self.h)
            self.h = None


class OracleModelB:
    FIELDS = ["x", "y", "z", "b", "mu_x", "mu_y", "mu_z", "metric"]

    def __init__(self, nx, ny, nz, edge, prm, conserved=False, bc=0, libm=False):
        self.n = nx * ny * nz
        self.shape = (nz, ny, nx)
        self.nb = ((nx - 1) // edge + 1) * ((ny - 1) // edge + 1) * (1 if nz == 1 else (nz - 1) // edge + 1)
        v = np.array([prm[k] for k in MODELB_KEYS], dtype=np.float64)
        self.h = lib().oracle_modelb_new(nx, ny, nz, edge, bc, dptr(v), int(libm), int(conserved))

    def init_mt(self, seed=1234, amp=0.05, z_amp=0.001):
        lib().oracle_modelb_init_mt(self.h, seed, amp, z_amp)

    def set_fields(self, x, y, z):
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z)]
        lib().oracle_modelb_set(self.h, dptr(a[0]), dptr(a[1]), dptr(a[2]))

    def step(self, n=1, mode=1):
        lib().oracle_modelb_step(self.h, n, mode)

    def field(self, name):
        out = np.empty(self.n)
        lib().oracle_modelb_get_field(self.h, self.FIELDS.index(name), dptr(out))
        return out.reshape(self.shape)

    def flags(self):
        w = np.empty(self.nb, np.int32); nx_ = np.empty(self.nb, np.int32)
        lib().oracle_modelb_get_flags(self.h, iptr(w), iptr(nx_))
        return w, nx_

    def last_avg(self):
        a = np.empty(3)
        lib().oracle_modelb_last_avg(self.h, dptr(a))
        return a

    def set_owned(self, ob0, ob1):
        """Slab runs: block rows [ob0, ob1) are own, the others ghosts."""
        lib().oracle_modelb_set_owned(self.h, int(ob0), int(ob1))

    def set_field(self, name, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        lib().oracle_modelb_set_field(self.h, self.FIELDS.index(name), dptr(a))

    def set_flags(self, wake):
        a = np.ascontiguousarray(wake, dtype=np.int32)
        lib().oracle_modelb_set_flags(self.h, iptr(a))

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_modelb_free(self.h)
            self.h = None


class OracleKH:
    FIELDS = ["Mass", "Momx", "Momy", "Energy", "rho", "p", "vx", "vy", "metric"]

    def __init__(self, nx, ny, edge, prm, conserved=False, bc=0):
        self.n = nx * ny
        self.shape = (1, ny, nx)
        self.nb = ((nx - 1) // edge + 1) * ((ny - 1) // edge + 1)
        v = np.array([prm[k] for k in KH_KEYS], dtype=np.float64)
        self.h = lib().oracle_kh_new(nx, ny, edge, bc, dptr(v), int(conserved))

    def init_smooth(self):
        lib().oracle_kh_init_smooth(self.h)

    def set_primitive(self, rho, p, vx, vy):
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (rho, p, vx, vy)]
        lib().oracle_kh_set_primitive(self.h, *[dptr(v) for v in a])

    def step(self, n=1, mode=1):
        lib().oracle_kh_step(self.h, n, mode)

    def field(self, name):
        out = np.empty(self.n)
        lib().oracle_kh_get_field(self.h, self.FIELDS.index(name), dptr(out))
        return out.reshape(self.shape)

    def flags(self):
        w = np.empty(self.nb, np.int32); nx_ = np.empty(self.nb, np.int32)
        lib().oracle_kh_get_flags(self.h, iptr(w), iptr(nx_))
        return w, nx_

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_kh_free(self.h)
            self.h = None


def tip_profile(f, dz=40):
    """Extract_Tip restated (oracle): f is (nz, ny, nx)."""
    nz, ny, nx = f.shape
    f = np.ascontiguousarray(f, dtype=np.float64)
    tip = np.zeros(dz + 1, np.int32)
    m = ctypes.c_int()
    lib().oracle_tip_profile(dptr(f), nx, ny, nz, dz, iptr(tip), ctypes.byref(m))
    return tip, m.value


def size_distribution(f, cap=1 << 20):
    """coarsening_analysis restated (oracle): (avg, volume, island sizes in scan order)."""
    nz, ny, nx = f.shape
    f = np.ascontiguousarray(f, dtype=np.float64)
    sizes = np.zeros(cap, np.int64)
    avg = ctypes.c_double()
    vol = ctypes.c_long()
    n = lib().oracle_size_distribution(dptr(f), nx, ny, nz, ctypes.byref(avg), ctypes.byref(vol),
                                       sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), cap)
    return avg.value, vol.value, sizes[:min(n, cap)].copy()
