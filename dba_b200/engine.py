"""ctypes binding of include/dba.h and a small Simulation wrapper.

The wrapper mirrors the reference programs' life cycle (ReadInput, Allocate,
Initialize, time loop, output) one call per stage; see include/dba.h for the
reference function each entry point replaces.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))

MODELS = {"dendrite": 0, "modelb": 1, "kh": 2}
FIELDS = {
    0: ["p", "T"],
    1: ["x", "y", "z", "b", "mu_x", "mu_y", "mu_z"],
    2: ["Mass", "Momx", "Momy", "Energy", "rho", "p", "vx", "vy"],
}
OPT_WAIT_LIMIT = 1          # dba_set_option
BATCH_PERSISTENT = 1        # dba_batch_set_option
BATCH_WAIT_LIMIT = 2
DBA_ERR = {0: "ok", 1: "config", 2: "cuda", 3: "nomem", 4: "io", 5: "nonfinite", 6: "timeout", 7: "state", 8: "arg"}


class DBAError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        msg = _lib().dba_strerror(code).decode() if _LIB is not None else DBA_ERR.get(code, "?")
        super().__init__(f"{what}: DBA status {code} ({msg})")


_d, _i, _u64 = ctypes.c_double, ctypes.c_int, ctypes.c_ulonglong


class Config(ctypes.Structure):
    _fields_ = [
        ("model", _i), ("nx", _i), ("ny", _i), ("nz", _i), ("t_total", _i), ("t_freq", _i), ("mode", _i),
        ("dt", _d), ("dx", _d), ("dy", _d), ("dz", _d),
        ("delta", _d), ("tau", _d), ("epsilon", _d), ("alpha", _d), ("gamma", _d), ("Delta", _d),
        ("metric_p", _d), ("metric_T", _d),
        ("chi_xy", _d), ("chi_xz", _d), ("chi_yz", _d), ("chi_xb", _d), ("chi_yb", _d), ("chi_zb", _d),
        ("vx", _i), ("vy", _i), ("vz", _i), ("rx", _i), ("ry", _i), ("rz", _i), ("n", _i), ("m", _i),
        ("eps_x", _d), ("eps_y", _d), ("eps_z", _d), ("eps_phi", _d),
        ("mob_x", _d), ("mob_y", _d), ("mob_z", _d), ("mob_phi", _d),
        ("x0", _d), ("y0", _d), ("z0", _d), ("K", _d), ("z_crit", _d), ("p_gel", _d), ("k_0", _d),
        ("metric_eps", _d), ("kh_gamma", _d),
        ("block", _i), ("precision", _i), ("bc", _i), ("conserved", _i), ("ic", _i),
        ("seed", _u64), ("ic_radius", _d), ("ic_width", _d), ("ic_corner", _i),
        ("noise_amp", _d), ("noise_amp_z", _d), ("tiles", _i), ("cfl", _d),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Obs(ctypes.Structure):
    _fields_ = [("step", ctypes.c_long), ("time", _d), ("active_blocks", _i * 2), ("total_blocks", _i),
                ("tip", _d), ("integral", _d * 4), ("vy_mode", _d), ("cell_updates", ctypes.c_long), ("dt", _d)]


class Info(ctypes.Structure):
    _fields_ = [("nbx", _i), ("nby", _i), ("nbz", _i), ("nb", _i), ("dims", _i), ("nfields", _i),
                ("nchannels", _i), ("device_bytes", ctypes.c_size_t), ("step", ctypes.c_long), ("grid_ctas", _i),
                ("active_block_steps", ctypes.c_long), ("cells_per_block", ctypes.c_long)]


class Prof(ctypes.Structure):
    _fields_ = [("steps", _i), ("step_ms", _d), ("stencil_ms", _d), ("reduce_ms", _d), ("correct_ms", _d),
                ("active_blocks", ctypes.c_long), ("active_blocks_ch", ctypes.c_long * 2),
                ("ch0_only_blocks", ctypes.c_long), ("cells_per_block", ctypes.c_long)]


class BatchConfig(ctypes.Structure):
    _fields_ = [("precision", _i), ("block", _i), ("max_slots", _i), ("block_capacity", _i),
                ("cell_capacity", ctypes.c_size_t), ("threads", _i)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("free_cells", ctypes.c_size_t), ("largest_free_cells", ctypes.c_size_t),
                ("free_blocks", ctypes.c_long), ("largest_free_blocks", ctypes.c_long), ("live_slots", _i),
                ("step", ctypes.c_long), ("active_block_steps", ctypes.c_long), ("grid_ctas", _i)]


_LIB = None


def lib_path():
    return os.path.join(_HERE, "libdba_b200.so")


def load_library():
    """Load libdba_b200.so (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        path = lib_path()
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build it with `python dba_b200/build.py`")
        L = ctypes.CDLL(path)
        P, V = ctypes.POINTER, ctypes.c_void_p
        sig = {
            "dba_config_default": (_i, [_i, P(Config)]),
            "dba_parse_input": (_i, [ctypes.c_char_p, _i, P(Config)]),
            "dba_create": (_i, [P(Config), P(V)]),
            "dba_init": (_i, [V, P(_d)]),
            "dba_step": (_i, [V, _i, _i]),
            "dba_sync": (_i, [V]),
            "dba_read_field": (_i, [V, _i, P(_d)]),
            "dba_read_field_f32": (_i, [V, _i, P(ctypes.c_float)]),
            "dba_init_f32": (_i, [V, P(ctypes.c_float)]),
            "dba_read_flags": (_i, [V, _i, P(ctypes.c_int32)]),
            "dba_observables": (_i, [V, P(Obs)]),
            "dba_tip": (_i, [V, P(_d)]),
            "dba_write_vtk": (_i, [V, ctypes.c_char_p]),
            "dba_write_active_vtk": (_i, [V, ctypes.c_char_p]),
            "dba_checkpoint": (_i, [V, ctypes.c_char_p]),
            "dba_restore": (_i, [V, ctypes.c_char_p]),
            "dba_get_info": (_i, [V, P(Info)]),
            "dba_get_config": (_i, [V, P(Config)]),
            "dba_destroy": (None, [V]),
            "dba_strerror": (ctypes.c_char_p, [_i]),
            "dba_struct_size": (ctypes.c_size_t, [_i]),
            "dba_tip_profile": (_i, [V, _i, _i, P(_i), P(_i)]),
            "dba_write_vtr": (_i, [V, ctypes.c_char_p, _i, _i]),
            "dba_wait_io": (_i, [V]),
            "dba_size_distribution": (_i, [V, _i, P(_d), P(ctypes.c_long), P(ctypes.c_long), P(ctypes.c_long),
                                           ctypes.c_long]),
            "dba_step_profiled": (_i, [V, _i, _i, P(Prof)]),
            "dba_get_stream": (_i, [V, P(V)]),
            "dba_state_size": (_i, [V, P(ctypes.c_size_t)]),
            "dba_save_state": (_i, [V, V, ctypes.c_size_t]),
            "dba_load_state": (_i, [V, V, ctypes.c_size_t]),
            "dba_batch_create": (_i, [P(BatchConfig), P(V)]),
            "dba_batch_add": (_i, [V, P(Config), P(_d), P(_i)]),
            "dba_batch_remove": (_i, [V, _i]),
            "dba_batch_step": (_i, [V, _i]),
            "dba_batch_sync": (_i, [V]),
            "dba_batch_tips": (_i, [V, P(_d), P(ctypes.c_long)]),
            "dba_batch_read_field": (_i, [V, _i, _i, P(_d)]),
            "dba_batch_get_info": (_i, [V, P(BatchInfo)]),
            "dba_batch_get_stream": (_i, [V, P(V)]),
            "dba_batch_destroy": (None, [V]),
            "dba_batch_set_option": (_i, [V, _i, ctypes.c_longlong]),
            "dba_set_option": (_i, [V, _i, ctypes.c_longlong]),
            "dba_rows_pack": (_i, [V, _i, _i, V]),
            "dba_rows_unpack": (_i, [V, _i, _i, V]),
            "dba_flag_rows": (_i, [V, _i, _i, _i, V]),
            "dba_slab_rows": (_i, [V, _i, _i, ctypes.c_longlong]),
            "dba_lazy_change": (_i, [V, _i, V]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        for k, cls in ((0, Config), (1, Obs), (2, Info), (3, Prof)):
            if L.dba_struct_size(k) != ctypes.sizeof(cls):
                raise RuntimeError(f"struct layout mismatch for {cls.__name__}")
        _LIB = L
    return _LIB


def _lib():
    return load_library()


def _check(code, what):
    if code != 0:
        raise DBAError(code, what)


def config(model, **overrides):
    """dba_config_default(model) with fields overridden by keyword."""
    m = MODELS[model] if isinstance(model, str) else int(model)
    c = Config()
    _check(_lib().dba_config_default(m, ctypes.byref(c)), "dba_config_default")
    for k, v in overrides.items():
        if not hasattr(c, k):
            raise KeyError(k)
        setattr(c, k, v)
    return c


def parse_input(path, model):
    m = MODELS[model] if isinstance(model, str) else int(model)
    c = Config()
    _check(_lib().dba_parse_input(str(path).encode(), m, ctypes.byref(c)), f"dba_parse_input({path})")
    return c


def _buf(buf):
    if isinstance(buf, np.ndarray):
        return ctypes.c_void_p(buf.ctypes.data), buf.nbytes
    # torch tensor (e.g. pinned host memory)
    return ctypes.c_void_p(buf.data_ptr()), buf.numel() * buf.element_size()


class Simulation:
    """One engine context on the current CUDA device."""

    def __init__(self, cfg):
        self._L = _lib()
        self.cfg = cfg
        self._h = ctypes.c_void_p()
        _check(self._L.dba_create(ctypes.byref(cfg), ctypes.byref(self._h)), "dba_create")
        self.shape = (cfg.nz, cfg.ny, cfg.nx)
        self.n = cfg.nx * cfg.ny * cfg.nz
        self.fields = FIELDS[cfg.model]
        self.info = self.get_info()

    def get_info(self):
        inf = Info()
        _check(self._L.dba_get_info(self._h, ctypes.byref(inf)), "dba_get_info")
        return inf

    def init(self, ic=None):
        if ic is None:
            _check(self._L.dba_init(self._h, None), "dba_init")
        else:
            a = np.ascontiguousarray(np.concatenate([np.asarray(f, np.float64).ravel() for f in ic]))
            _check(self._L.dba_init(self._h, a.ctypes.data_as(ctypes.POINTER(_d))), "dba_init")
        return self

    def init_f32(self, ic):
        """dba_init from FP32 host fields: `ic` is a C-contiguous float32 array holding the
        initial fields one after another (dendrite p, T; Model B x, y, z; KH rho, p, vx, vy),
        for instance page-locked memory, which the device copies from at full link speed."""
        nic = {0: 2, 1: 3, 2: 4}[self.cfg.model]
        if ic.dtype != np.float32 or not ic.flags.c_contiguous or ic.size != nic * self.n:
            raise ValueError("ic must be a C-contiguous float32 array of the initial fields")
        _check(self._L.dba_init_f32(self._h, ic.ctypes.data_as(ctypes.POINTER(ctypes.c_float))), "dba_init_f32")
        return self

    def field_f32(self, name, out=None):
        """Current values of a field rounded to float32 (dba_read_field_f32), shape (nz, ny, nx);
        `out` as in field() but float32."""
        fid = self._fid(name)
        if out is None:
            out = np.empty(self.n, np.float32)
        elif out.dtype != np.float32 or out.size != self.n or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float32 array of %d elements" % self.n)
        _check(self._L.dba_read_field_f32(self._h, fid, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
               "dba_read_field_f32")
        return out.reshape(self.shape)

    def step(self, n=1, mode=1):
        _check(self._L.dba_step(self._h, int(n), int(mode)), "dba_step")

    def sync(self):
        _check(self._L.dba_sync(self._h), "dba_sync")

    def _fid(self, name):
        return self.fields.index(name) if isinstance(name, str) else int(name)

    def field(self, name, out=None):
        """Current values of a field as float64, shape (nz, ny, nx).  `out`, if given,
        is a C-contiguous float64 array of nx*ny*nz elements that receives them (for
        instance page-locked host memory, which the device copies into at full link
        speed) and is returned reshaped."""
        fid = self._fid(name)
        if out is None:
            out = np.empty(self.n, np.float64)
        elif out.dtype != np.float64 or out.size != self.n or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of %d elements" % self.n)
        _check(self._L.dba_read_field(self._h, fid, out.ctypes.data_as(ctypes.POINTER(_d))), "dba_read_field")
        return out.reshape(self.shape)

    def flags(self, which=0):
        out = np.empty(self.info.nb, np.int32)
        _check(self._L.dba_read_flags(self._h, int(which), out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))),
               "dba_read_flags")
        return out

    def cell_updates(self):
        """Active cell-updates (cells of blocks active in any channel) since init."""
        inf = self.get_info()
        return inf.active_block_steps * inf.cells_per_block

    def tip(self):
        v = _d()
        _check(self._L.dba_tip(self._h, ctypes.byref(v)), "dba_tip")
        return v.value

    def observables(self):
        o = Obs()
        _check(self._L.dba_observables(self._h, ctypes.byref(o)), "dba_observables")
        return {"step": o.step, "time": o.time, "active_blocks": list(o.active_blocks), "total_blocks": o.total_blocks,
                "tip": o.tip, "integral": list(o.integral), "vy_mode": o.vy_mode, "cell_updates": o.cell_updates,
                "dt": o.dt}

    def write_vtr(self, base, pieces=1, binary=True, background=False):
        """VTK XML RectilinearGrid output: <base>.vtr, or <base>_<r>.vtr pieces and <base>.pvtr."""
        flags = (1 if binary else 0) | (2 if background else 0)
        _check(self._L.dba_write_vtr(self._h, str(base).encode(), int(pieces), flags), "dba_write_vtr")

    def wait_io(self):
        """Join background writers; raises the first write error."""
        _check(self._L.dba_wait_io(self._h), "dba_wait_io")

    def tip_profile(self, dz=40, field=0):
        """Extract_Tip on the device: (tip_x[0..dz], tip_x_max) for planes Nz/2 .. Nz/2+dz."""
        tip = np.zeros(dz + 1, np.int32)
        m = _i()
        _check(self._L.dba_tip_profile(self._h, int(self._fid(field)), int(dz),
                                       tip.ctypes.data_as(ctypes.POINTER(_i)), ctypes.byref(m)), "dba_tip_profile")
        return tip, m.value

    def size_distribution(self, field, max_sizes=1 << 16):
        """coarsening_analysis on the device: (avg, volume, island sizes in scan order)."""
        fid = int(self._fid(field))
        avg, vol, nis = _d(), ctypes.c_long(), ctypes.c_long()
        sizes = np.zeros(max(1, max_sizes), np.int64)
        st = self._L.dba_size_distribution(self._h, fid, ctypes.byref(avg), ctypes.byref(vol), ctypes.byref(nis),
                                           sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), int(max_sizes))
        if st == 8 and nis.value > max_sizes:       # too many islands for the buffer: retry once, sized
            return self.size_distribution(field, int(nis.value))
        _check(st, "dba_size_distribution")
        return avg.value, vol.value, sizes[:nis.value].copy()

    def rows_pack(self, row0, nrows, dev_ptr):
        _check(self._L.dba_rows_pack(self._h, int(row0), int(nrows), ctypes.c_void_p(dev_ptr)), "dba_rows_pack")

    def rows_unpack(self, row0, nrows, dev_ptr):
        _check(self._L.dba_rows_unpack(self._h, int(row0), int(nrows), ctypes.c_void_p(dev_ptr)), "dba_rows_unpack")

    def flag_rows(self, op, brow0, nbrows, dev_ptr=0):
        _check(self._L.dba_flag_rows(self._h, int(op), int(brow0), int(nbrows), ctypes.c_void_p(dev_ptr)),
               "dba_flag_rows")

    def slab_rows(self, first_block_row, block_rows, domain_cells):
        """dba_slab_rows: the context is a slab of a larger Model B domain; block rows
        [first, first + count) are its own, the others ghosts."""
        _check(self._L.dba_slab_rows(self._h, int(first_block_row), int(block_rows), int(domain_cells)),
               "dba_slab_rows")

    def lazy_change(self, op, ptr):
        """dba_lazy_change: the last step's fixed-point change totals to (op 0) or from (op 1) ptr."""
        _check(self._L.dba_lazy_change(self._h, int(op), ctypes.c_void_p(ptr)), "dba_lazy_change")

    def set_option(self, option, value):
        """dba_set_option: OPT_WAIT_LIMIT bounds the device retry loops (post-processing)."""
        _check(self._L.dba_set_option(self._h, int(option), int(value)), "dba_set_option")

    def step_profiled(self, n, mode=1):
        p = Prof()
        _check(self._L.dba_step_profiled(self._h, int(n), int(mode), ctypes.byref(p)), "dba_step_profiled")
        return {k: (list(getattr(p, k)) if k == "active_blocks_ch" else getattr(p, k)) for k, _ in p._fields_}

    @property
    def stream(self):
        v = ctypes.c_void_p()
        _check(self._L.dba_get_stream(self._h, ctypes.byref(v)), "dba_get_stream")
        return v.value or 0

    def state_size(self):
        n = ctypes.c_size_t()
        _check(self._L.dba_state_size(self._h, ctypes.byref(n)), "dba_state_size")
        return n.value

    def save_state(self, buf):
        """buf: a writable host buffer (numpy uint8 array or pinned torch tensor data_ptr holder)."""
        ptr, size = _buf(buf)
        _check(self._L.dba_save_state(self._h, ptr, size), "dba_save_state")

    def load_state(self, buf):
        ptr, size = _buf(buf)
        _check(self._L.dba_load_state(self._h, ptr, size), "dba_load_state")

    def write_vtk(self, path):
        _check(self._L.dba_write_vtk(self._h, str(path).encode()), "dba_write_vtk")

    def write_active_vtk(self, path):
        _check(self._L.dba_write_active_vtk(self._h, str(path).encode()), "dba_write_active_vtk")

    def checkpoint(self, path):
        _check(self._L.dba_checkpoint(self._h, str(path).encode()), "dba_checkpoint")

    def restore(self, path):
        _check(self._L.dba_restore(self._h, str(path).encode()), "dba_restore")

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._L.dba_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Batch:
    """Many independent 2-D dendrite simulations advanced by one kernel per step
    (include/dba.h, dba_batch_*).  Slots are admitted while the batch's device
    arena and block space have room and retired when done."""

    def __init__(self, precision=1, block=8, max_slots=64, block_capacity=1 << 16, cell_capacity=0, threads=256):
        self._L = _lib()
        self.cfg = BatchConfig(precision, block, max_slots, block_capacity, cell_capacity, threads)
        self._h = ctypes.c_void_p()
        _check(self._L.dba_batch_create(ctypes.byref(self.cfg), ctypes.byref(self._h)), "dba_batch_create")
        self.max_slots = max_slots
        self.shapes = {}

    def add(self, cfg, ic=None):
        """Admit a simulation; returns its slot, or None when there is no room."""
        slot = _i()
        ptr = None
        if ic is not None:
            a = np.ascontiguousarray(np.concatenate([np.asarray(f, np.float64).ravel() for f in ic]))
            ptr = a.ctypes.data_as(ctypes.POINTER(_d))
        st = self._L.dba_batch_add(self._h, ctypes.byref(cfg), ptr, ctypes.byref(slot))
        if st == 3:
            return None
        _check(st, "dba_batch_add")
        self.shapes[slot.value] = (cfg.ny, cfg.nx)
        return slot.value

    def remove(self, slot):
        _check(self._L.dba_batch_remove(self._h, int(slot)), "dba_batch_remove")
        self.shapes.pop(slot, None)

    def step(self, n):
        _check(self._L.dba_batch_step(self._h, int(n)), "dba_batch_step")

    def sync(self):
        _check(self._L.dba_batch_sync(self._h), "dba_batch_sync")

    def set_option(self, option, value):
        """dba_batch_set_option: BATCH_PERSISTENT (1 persistent launches, 0 one launch per
        step) or BATCH_WAIT_LIMIT (polls per grid-barrier wait before DBA_ERR_TIMEOUT)."""
        _check(self._L.dba_batch_set_option(self._h, int(option), int(value)), "dba_batch_set_option")

    def tips(self):
        t = np.empty(self.max_slots, np.float64)
        s = np.empty(self.max_slots, np.int64)
        _check(self._L.dba_batch_tips(self._h, t.ctypes.data_as(ctypes.POINTER(_d)),
                                      s.ctypes.data_as(ctypes.POINTER(ctypes.c_long))), "dba_batch_tips")
        return t, s

    def field(self, slot, name):
        fid = ["p", "T"].index(name) if isinstance(name, str) else int(name)
        ny, nx = self.shapes[slot]
        out = np.empty(ny * nx, np.float64)
        _check(self._L.dba_batch_read_field(self._h, int(slot), fid, out.ctypes.data_as(ctypes.POINTER(_d))),
               "dba_batch_read_field")
        return out.reshape(1, ny, nx)

    def info(self):
        inf = BatchInfo()
        _check(self._L.dba_batch_get_info(self._h, ctypes.byref(inf)), "dba_batch_get_info")
        return inf

    @property
    def stream(self):
        v = ctypes.c_void_p()
        _check(self._L.dba_batch_get_stream(self._h, ctypes.byref(v)), "dba_batch_get_stream")
        return v.value or 0

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._L.dba_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
