"""ctypes binding of the C ABI declared in include/rhgpu.h.

The same entry-point set is exported under three prefixes:
  rhgpu_  the B200 library (rhybrid_b200/librhgpu.so, the product),
  rho_    the C restatement of the reference algorithm (oracle, tests only),
  rhref_  the reference's own sources built against the oracle shim (tests only).
`Library` binds any of them; the package itself only ever loads rhgpu_.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

# rhgpu.h: particle paths
PATH_FAST = 0
PATH_EXACT = 1
PATH_FP32 = 2

# rhgpu.h: learned denoiser parameter count
DN_PARAMS = 20784

# rhgpu.h: status codes
OK, ERR_ARG, ERR_CUDA, ERR_STATE, ERR_DEVICE, ERR_NOMEM, ERR_CAPACITY = range(7)

# rhgpu.h: device error bits
DEVERR_NAN_PARTICLE = 1
DEVERR_FAST_PARTICLE = 2
DEVERR_CAPACITY = 4

# rhgpu.h: cell flag bits
FLAG_INNER_FIELD = 1
FLAG_INNER_NODE = 2
FLAG_INNER_PARTICLE = 4
FLAG_INNER_CELLEP = 8

# rhgpu.h: rhgpu_array_id
ARRAYS = [
    "faceB", "cellB", "cellUe", "cellEp", "cellRhoQi", "cellJi", "cellJ",
    "nodeRhoQi", "nodeJi", "nodeJ", "nodeUe", "nodeB", "nodeE", "nodeEta", "cellAverageB",
]
ARRAY_ID = {n: i for i, n in enumerate(ARRAYS)}
SCALAR_ARRAYS = {"cellRhoQi", "nodeRhoQi", "nodeEta"}

# rhgpu.h: rhgpu_counter_id
FIELD_COUNTERS = [
    "fieldMinCellRhoQi", "fieldMaxCellUe", "fieldMaxNodeUe", "fieldMaxVw", "fieldMaxE",
    "fieldMinNodeRhoQi", "gridTemporalAverageCounter",
]
SPECIES_COUNTERS = ["particleMaxVi", "particleEscape", "particleEscapeKineticEnergy",
                    "particleImpact", "particleImpactKineticEnergy"]

# rhgpu.h: rhgpu_reduce_diagnostics layout
DIAG_PARTICLE = ["N_macroParticles", "N_realParticles", "sumVx", "sumVy", "sumVz", "sumV", "sumWV2", "maxVi"]
DIAG_FIELD = ["N_cells", "sumBx", "sumBy", "sumBz", "sumB", "maxB", "sumDivB", "maxDivB", "maxDivBPerB", "sumB2",
              "sumCellJix", "sumCellJiy", "sumCellJiz", "sumCellJi", "maxCellJi",
              "sumCellEpx", "sumCellEpy", "sumCellEpz", "sumCellEp", "maxCellEp", "sumCellEp2",
              "sumNodeEx", "sumNodeEy", "sumNodeEz", "sumNodeE", "maxNodeE", "sumNodeE2",
              "sumCellE2", "maxUe", "sumCellRhoQi"]
# rhgpu_download_grid_counters planes (the reference's gridCounter* arrays)
GRID_COUNTERS = ["cellMaxUe", "cellMaxVi", "cellMinRhoQi", "nodeMaxE", "nodeMaxVw"]
# the six scales that follow with n >= 8*n_species + 36 (LogDataField names)
DIAG_SCALES = ["minInerLengthElectron", "maxInerLengthElectron", "minInerLengthProton", "maxInerLengthProton",
               "minTLarmor", "maxVAlfven"]

# rhgpu.h: physical constants
PERMEABILITY = 1.2566370614359173e-06
CHARGE_ELEMENTARY = 1.602176634e-19
MASS_PROTON = 1.67262192369e-27
MASS_ELECTRON = 9.1093837015e-31
PERMITTIVITY = 8.8541878128e-12
BOLTZMANN = 1.380649e-23
GRAVITY = 6.67430e-11


class Params(C.Structure):
    """struct rhgpu_params"""
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("periodic", C.c_int32 * 3),
        ("x_min", C.c_double), ("y_min", C.c_double), ("z_min", C.c_double),
        ("dx", C.c_double), ("dt", C.c_double), ("t_initial", C.c_double),
        ("use_hall", C.c_int32), ("use_electron_pressure", C.c_int32),
        ("isothermal_electrons", C.c_int32), ("use_gravity", C.c_int32),
        ("use_initial_flow_through", C.c_int32), ("n_linear_smoothings_nodeE", C.c_int32),
        ("use_gaussian_smoothing_nodeE", C.c_int32), ("reserved0", C.c_int32),
        ("electron_pressure_coeff", C.c_double),
        ("gaussian_coeffs", C.c_double * 4),
        ("field_obstacle_Ue", C.c_double * 3),
        ("GMdt", C.c_double),
        ("max_ion_speed2", C.c_double),
        ("max_electron_speed2", C.c_double),
        ("min_ion_charge_density", C.c_double),
        ("max_electric_field2", C.c_double),
        ("max_whistler_speed", C.c_double),
        ("initial_flow_through_period", C.c_double),
        ("imf_B", C.c_double * 3),
        ("imf_boundary_cellB", C.c_int32 * 6),
        ("imf_boundary_faceB", C.c_int32 * 6),
    ]


class Species(C.Structure):
    """struct rhgpu_species"""
    _fields_ = [
        ("q", C.c_double), ("m", C.c_double), ("R2_obstacle", C.c_double),
        ("accumulate", C.c_int32), ("accelerate", C.c_int32),
    ]


class RhError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"status {code}: {msg}")
        self.code = code


_P = C.c_void_p
_D = C.POINTER(C.c_double)
_U32 = C.POINTER(C.c_uint32)
_U8 = C.POINTER(C.c_uint8)
_I64 = C.POINTER(C.c_int64)

# entry point -> argtypes (all return int32 status unless listed in _RESTYPES)
_SIGNATURES = {
    "create": [C.POINTER(Params), C.c_int32, C.POINTER(Species), _I64, C.c_int32, C.POINTER(_P)],
    "destroy": [_P],
    "upload_array": [_P, C.c_int32, _D],
    "download_array": [_P, C.c_int32, _D],
    "upload_cell_flags": [_P, _U8],
    "upload_particles": [_P, C.c_int32, _U32, _D, C.c_int64],
    "num_particles": [_P, C.c_int32, _I64],
    "download_particles": [_P, C.c_int32, _U32, _D, C.c_int64, _I64],
    "step": [_P, C.c_int32],
    "push": [_P],
    "accumulate": [_P],
    "apply_boundaries": [_P],
    "propagate_fields": [_P],
    "get_counters": [_P, _D, C.c_int32],
    "get_time": [_P, _D, _I64],
    "last_error": [],
}
_OPTIONAL = {
    # the FP32 form's own particle records (GPU library only)
    "upload_particles_f32": [_P, C.c_int32, _U32, C.POINTER(C.c_float), C.c_int64, C.c_double],
    "download_particles_f32": [_P, C.c_int32, _U32, C.POINTER(C.c_float), C.c_int64, _I64, _D],
    "device_errors": [_P, _U32],
    "reduce_diagnostics": [_P, _D, C.c_int32],
    "fill_uniform": [_P, C.c_int32, C.c_void_p, C.c_void_p],
    "dn_add_crops": [_P, _P, C.c_int32, C.c_int32, C.c_int32, C.c_void_p],
    "dn_set_loss_border": [_P, C.c_int32],
    "dn_set_velocity_form": [_P, C.c_int32],
    "dn_set_keep_mask": [_P, C.c_void_p],
    "set_timing": [_P, C.c_int32],
    "get_timing": [_P, C.c_char_p, C.c_int32, _D, C.c_int32, C.POINTER(C.c_int32)],
    "last_launch_count": [_P, _I64],
    "stream": [_P],
    "version": [],
    "set_deposit_order": [_P, C.c_int32],
    "set_path": [_P, C.c_int32],
    "accumulate_noalloc": [_P],
    "dn_create": [C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.c_int32, C.POINTER(_P)],
    "dn_destroy": [_P],
    "dn_set_params": [_P, C.POINTER(C.c_float), C.c_int64],
    "dn_get_params": [_P, C.POINTER(C.c_float), C.c_int64],
    "dn_set_scales": [_P, C.c_double, C.c_double],
    "dn_apply": [_P, _D, _D, _D, _D, C.c_double],
    "dn_loss_grad": [_P, _D, _D, _D, _D, _D, C.POINTER(C.c_float)],
    "dn_add_pair": [_P, _P, C.c_int32, C.c_int32],
    "dn_train": [_P, C.c_int32, C.c_float, _D],
    "dn_pair_error": [_P, C.c_int32, _D],
    "dn_num_pairs": [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)],
    "set_denoiser": [_P, _P, C.c_int32],
    "set_threads": [_P, C.c_int32],
    "set_injectors": [_P, C.c_int32, C.c_void_p],
    "get_injection_counters": [_P, _D, C.c_int32],
    "source_rates": [_P, C.c_int32, _D],
    "philox4x32": [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)],
    "neutral_density": [C.c_void_p, C.c_double, C.c_int64, _D, _D, C.c_int32],
    "log_open": [_P, C.c_void_p],
    "log_write": [_P, C.c_int32, C.POINTER(C.c_int32), C.c_char_p, C.c_int32],
    "log_close": [_P],
    "set_population_averages": [_P, C.c_int32, C.POINTER(C.c_int32)],
    "set_grid_counters": [_P, C.c_int32],
    "download_grid_counters": [_P, _D],
    "output_averages": [_P, _D, _D, _D],
}
_RESTYPES = {"last_error": C.c_char_p, "version": C.c_char_p, "stream": C.c_void_p, "philox4x32": None}

INJECT_SOLARWIND = 1
INJECT_FLOW = 2
INJECT_EXOSPHERE = 3
INJECT_IONOSPHERE = 4
INJECT_CHAPMAN_IONOSPHERE = 5
IONO_PROFILES = {"ionoCosSzaDayConstantNight": 1, "ionoConstantDayConstantNight": 2, "ionoConstant": 3,
                 "ionoPolarCap": 4}
NEUTRAL_PROFILES = {"ChamberlainH": 1, "ChamberlainT": 2, "Exponential": 3, "PowerLaw": 4, "VenusHydrogen": 5,
                    "VenusOxygen": 6, "MercurySodiumExner20": 7}
# flow injector walls (rhgpu_injector.inflow_walls)
WALLS = {"+x": 1, "-x": 2, "+y": 4, "-y": 8, "+z": 16, "-z": 32}


class Injector(C.Structure):
    """rhgpu_injector: one particle source (the reference's solar wind or flow injector)."""
    _fields_ = [("species", C.c_int32), ("type", C.c_int32), ("velocity", C.c_double * 3),
                ("density", C.c_double), ("temperature", C.c_double), ("macroparticles_per_cell", C.c_double),
                ("inflow_walls", C.c_int32), ("reserved", C.c_int32), ("seed", C.c_uint64),
                ("profile", C.c_int32), ("n_components", C.c_int32), ("r0", C.c_double),
                ("n0", C.c_double * 4), ("H0", C.c_double * 4), ("T0", C.c_double * 4), ("k0", C.c_double * 4),
                ("gm_object", C.c_double), ("exobase_radius", C.c_double), ("shadow_radius", C.c_double),
                ("ionization_rate", C.c_double), ("ionization_factor_shadow", C.c_double),
                ("total_production_rate", C.c_double), ("macroparticles_per_cell_relative", C.c_double),
                ("upstream_macro_ratio", C.c_double), ("emission_radius", C.c_double),
                ("noon_factor", C.c_double), ("night_factor", C.c_double), ("iono_profile", C.c_int32),
                ("reserved2", C.c_int32)]


class LogConfig(C.Structure):
    """rhgpu_log_config: where and how the population and field logs are written."""
    _fields_ = [("directory", C.c_char_p), ("species_names", C.POINTER(C.c_char_p)), ("precision", C.c_int32),
                ("include_inner_cells", C.c_int32), ("max_B_stop_run", C.c_double)]


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


class Library:
    """A loaded implementation of the rhgpu C ABI under some prefix."""

    def __init__(self, path: str, prefix: str):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.path = path
        self.prefix = prefix
        self.dll = C.CDLL(path)
        self.fn = {}
        for name, argt in list(_SIGNATURES.items()) + list(_OPTIONAL.items()):
            sym = prefix + name
            if not hasattr(self.dll, sym):
                if name in _SIGNATURES:
                    raise RuntimeError(f"{path}: missing symbol {sym}")
                continue
            f = getattr(self.dll, sym)
            f.argtypes = argt
            f.restype = _RESTYPES.get(name, C.c_int32)
            self.fn[name] = f

    def has(self, name: str) -> bool:
        return name in self.fn

    def last_error(self) -> str:
        s = self.fn["last_error"]()
        return s.decode() if s else ""

    def call(self, name: str, *args) -> int:
        rc = self.fn[name](*args)
        if rc != OK:
            raise RhError(rc, f"{self.prefix}{name}: {self.last_error()}")
        return rc


class Context:
    """One simulation context of a Library (rhgpu_ctx*)."""

    def __init__(self, lib: Library, params: Params, species: list, capacity=None, device: int = 0):
        self.lib = lib
        self.params = params
        self.species = list(species)
        self.cell_flags = None           # the flags last given to upload_cell_flags
        self.injectors = []              # the sources last given to set_injectors
        self.nspecies = len(species)
        self.ncells = params.nx * params.ny * params.nz
        arr = (Species * len(species))(*species)
        cap = np.asarray(capacity if capacity is not None else [0] * len(species), dtype=np.int64)
        h = C.c_void_p()
        lib.call("create", C.byref(params), len(species), arr, _ptr(cap, C.c_int64), device, C.byref(h))
        self.h = h

    def close(self):
        if self.h:
            self.lib.call("destroy", self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # grid arrays -----------------------------------------------------
    def upload_array(self, name: str, data: np.ndarray):
        dim = 1 if name in SCALAR_ARRAYS else 3
        a = np.ascontiguousarray(data, dtype=np.float64).reshape(-1)
        if a.size != dim * self.ncells:
            raise ValueError(f"{name}: expected {dim * self.ncells} values, got {a.size}")
        self.lib.call("upload_array", self.h, ARRAY_ID[name], _ptr(a, C.c_double))

    def download_array(self, name: str) -> np.ndarray:
        dim = 1 if name in SCALAR_ARRAYS else 3
        out = np.empty(dim * self.ncells, dtype=np.float64)
        self.lib.call("download_array", self.h, ARRAY_ID[name], _ptr(out, C.c_double))
        return out if dim == 1 else out.reshape(self.ncells, 3)

    def upload_cell_flags(self, flags: np.ndarray):
        f = np.ascontiguousarray(flags, dtype=np.uint8).reshape(-1)
        assert f.size == self.ncells
        self.lib.call("upload_cell_flags", self.h, _ptr(f, C.c_uint8))
        self.cell_flags = f.copy()

    # particles -------------------------------------------------------
    def upload_particles(self, s: int, counts: np.ndarray, particles: np.ndarray):
        cnt = np.ascontiguousarray(counts, dtype=np.uint32)
        p = np.ascontiguousarray(particles, dtype=np.float64).reshape(-1, 7)
        assert cnt.size == self.ncells
        self.lib.call("upload_particles", self.h, s, _ptr(cnt, C.c_uint32), _ptr(p, C.c_double), p.shape[0])

    def num_particles(self, s: int) -> int:
        n = C.c_int64()
        self.lib.call("num_particles", self.h, s, C.byref(n))
        return n.value

    def download_particles(self, s: int):
        n = self.num_particles(s)
        cnt = np.empty(self.ncells, dtype=np.uint32)
        p = np.empty((max(n, 1), 7), dtype=np.float64)
        nout = C.c_int64()
        self.lib.call("download_particles", self.h, s, _ptr(cnt, C.c_uint32), _ptr(p, C.c_double), p.shape[0],
                      C.byref(nout))
        return cnt, p[: nout.value]

    def upload_particles_f32(self, s: int, counts: np.ndarray, particles: np.ndarray, weight: float):
        """FP32 form only: particles as 6 float32 per record (offsets in the
        cell in units of dx, in [0, 1), then the velocity), the species' weight
        apart (rhgpu_upload_particles_f32)."""
        cnt = np.ascontiguousarray(counts, dtype=np.uint32)
        p = np.ascontiguousarray(particles, dtype=np.float32).reshape(-1, 6)
        assert cnt.size == self.ncells
        self.lib.call("upload_particles_f32", self.h, s, _ptr(cnt, C.c_uint32), _ptr(p, C.c_float), p.shape[0],
                      float(weight))

    def download_particles_f32(self, s: int):
        """FP32 form only: (counts, 6-float records, weight)."""
        n = self.num_particles(s)
        cnt = np.empty(self.ncells, dtype=np.uint32)
        p = np.empty((max(n, 1), 6), dtype=np.float32)
        nout = C.c_int64()
        w = np.zeros(1)
        self.lib.call("download_particles_f32", self.h, s, _ptr(cnt, C.c_uint32), _ptr(p, C.c_float), p.shape[0],
                      C.byref(nout), _ptr(w, C.c_double))
        return cnt, p[: nout.value], float(w[0])

    # stepping --------------------------------------------------------
    def step(self, n: int = 1):
        self.lib.call("step", self.h, n)

    def push(self):
        self.lib.call("push", self.h)

    def accumulate(self):
        self.lib.call("accumulate", self.h)

    def apply_boundaries(self):
        self.lib.call("apply_boundaries", self.h)

    def propagate_fields(self):
        self.lib.call("propagate_fields", self.h)

    def counters(self) -> dict:
        n = len(FIELD_COUNTERS) + len(SPECIES_COUNTERS) * self.nspecies
        out = np.zeros(n, dtype=np.float64)
        self.lib.call("get_counters", self.h, _ptr(out, C.c_double), n)
        d = {k: out[i] for i, k in enumerate(FIELD_COUNTERS)}
        for s in range(self.nspecies):
            for j, k in enumerate(SPECIES_COUNTERS):
                d[f"{k}[{s}]"] = out[len(FIELD_COUNTERS) + len(SPECIES_COUNTERS) * s + j]
        return d

    def time(self):
        t = C.c_double()
        ts = C.c_int64()
        self.lib.call("get_time", self.h, C.byref(t), C.byref(ts))
        return t.value, ts.value

    def device_errors(self) -> int:
        w = C.c_uint32()
        self.lib.call("device_errors", self.h, C.byref(w))
        return w.value

    def reduce_diagnostics(self, scales: bool = False) -> dict:
        """rhgpu_reduce_diagnostics: the population log per species and the field
        log (with `scales`, also the field log's spatial, temporal and velocity scales)."""
        n = 8 * self.nspecies + 30 + (6 if scales else 0)
        out = np.zeros(n, dtype=np.float64)
        self.lib.call("reduce_diagnostics", self.h, _ptr(out, C.c_double), n)
        pops = [dict(zip(DIAG_PARTICLE, out[8 * s:8 * s + 8])) for s in range(self.nspecies)]
        return {"populations": pops, "field": dict(zip(DIAG_FIELD + DIAG_SCALES, out[8 * self.nspecies:]))}

    def log_open(self, directory: str, species_names, precision: int = 10, include_inner_cells: bool = False,
                 max_B_stop_run: float = float("inf")):
        """rhgpu_log_open: pop<NNN>_<name>.log per species and field.log in `directory`."""
        names = (C.c_char_p * self.nspecies)(*[n.encode() for n in species_names])
        self._log_cfg = LogConfig(str(directory).encode(), names, precision, 1 if include_inner_cells else 0,
                                  max_B_stop_run)
        self._log_names = names
        self.lib.call("log_open", self.h, C.cast(C.byref(self._log_cfg), C.c_void_p))

    def log_write(self, main_log_diagnostics: bool = False):
        """rhgpu_log_write: one line per log file; returns (stop_run, main-log text)."""
        stop = C.c_int32()
        buf = C.create_string_buffer(1 << 14)
        self.lib.call("log_write", self.h, 1 if main_log_diagnostics else 0, C.byref(stop), buf, len(buf))
        return bool(stop.value), buf.value.decode()

    def log_close(self):
        self.lib.call("log_close", self.h)

    def set_population_averages(self, group_of_species):
        """rhgpu_set_population_averages: output population of each species (-1: none)."""
        g = np.ascontiguousarray(group_of_species, dtype=np.int32)
        self._avg_groups = int(g.max()) + 1 if g.size and g.max() >= 0 else 0
        self.lib.call("set_population_averages", self.h, self._avg_groups, _ptr(g, C.c_int32))

    def set_grid_counters(self, enable: bool = True):
        """rhgpu_set_grid_counters: per-cell constraint counters on (zeroed) or off."""
        self.lib.call("set_grid_counters", self.h, 1 if enable else 0)

    def grid_counters(self) -> dict:
        """rhgpu_download_grid_counters: the five per-cell counter planes by name."""
        out = np.zeros(len(GRID_COUNTERS) * self.ncells, dtype=np.float64)
        self.lib.call("download_grid_counters", self.h, _ptr(out, C.c_double))
        return {k: out[i * self.ncells:(i + 1) * self.ncells] for i, k in enumerate(GRID_COUNTERS)}

    def output_averages(self, cellB: bool = True, populations: bool = True) -> dict:
        """rhgpu_output_averages: cellBAverage (N x 3) and per output population
        n_ave (N) and v_ave (N x 3); the returned sums and the counter restart."""
        N = self.ncells
        out = {}
        b = np.zeros(3 * N) if cellB else None
        G = getattr(self, "_avg_groups", 0) if populations else 0
        n = np.zeros(G * N) if G else None
        v = np.zeros(3 * G * N) if G else None
        nul = C.POINTER(C.c_double)()
        self.lib.call("output_averages", self.h, _ptr(b, C.c_double) if b is not None else nul,
                      _ptr(n, C.c_double) if n is not None else nul, _ptr(v, C.c_double) if v is not None else nul)
        if b is not None:
            out["cellBAverage"] = b.reshape(N, 3)
        if G:
            out["n_ave"] = n.reshape(G, N)
            out["v_ave"] = v.reshape(G, N, 3)
        return out

    def set_timing(self, on: bool):
        self.lib.call("set_timing", self.h, 1 if on else 0)

    def timing(self) -> dict:
        names = C.create_string_buffer(4096)
        ms = np.zeros(64, dtype=np.float64)
        n = C.c_int32()
        self.lib.call("get_timing", self.h, names, 4096, _ptr(ms, C.c_double), 64, C.byref(n))
        keys = names.value.decode().split(",") if names.value else []
        return {k: ms[i] for i, k in enumerate(keys[: n.value])}

    def last_launch_count(self) -> int:
        n = C.c_int64()
        self.lib.call("last_launch_count", self.h, C.byref(n))
        return n.value

    def stream(self) -> int:
        return self.lib.fn["stream"](self.h) or 0

    def set_deposit_order(self, order: int):
        self.lib.call("set_deposit_order", self.h, order)

    def accumulate_noalloc(self):
        """rhgpu_accumulate_noalloc: the exact-path deposit without any device allocation."""
        self.lib.call("accumulate_noalloc", self.h)

    def set_injectors(self, injectors):
        """rhgpu_set_injectors: the particle sources (a list of Injector; empty: none)."""
        arr = (Injector * max(len(injectors), 1))(*injectors)
        self.lib.call("set_injectors", self.h, len(injectors), C.cast(arr, C.c_void_p))
        self.injectors = list(injectors)

    def fill_uniform(self, s: int, density: float, temperature: float, velocity, ppc: float, seed: int = 1,
                     region=None):
        """rhgpu_fill_uniform: replaces species s by a uniform fill generated on
        the GPU (InjectorUniform; fast path and FP32 form). region: (x_lo, x_hi,
        y_lo, y_hi, z_lo, z_hi) of the cell centres, or None for the whole box."""
        j = Injector(species=s, type=0, density=density, temperature=temperature, macroparticles_per_cell=ppc,
                     seed=seed)
        for a in range(3):
            j.velocity[a] = velocity[a]
        reg = None
        if region is not None:
            reg = np.ascontiguousarray(region, dtype=np.float64)
            assert reg.size == 6
        self.lib.call("fill_uniform", self.h, s, C.cast(C.byref(j), C.c_void_p),
                      reg.ctypes.data_as(C.c_void_p) if reg is not None else None)

    def source_rates(self, injector: int) -> np.ndarray:
        """rhgpu_source_rates: expected macroparticles per step in every cell
        of a rate-based source (exosphere, ionospheres); zeros otherwise."""
        out = np.zeros(self.ncells, dtype=np.float64)
        self.lib.call("source_rates", self.h, injector, _ptr(out, C.c_double))
        return out

    def injection_counters(self) -> list:
        """rhgpu_get_injection_counters: per species the injected weight,
        macroparticles and weight * v^2."""
        out = np.zeros(3 * self.nspecies, dtype=np.float64)
        self.lib.call("get_injection_counters", self.h, _ptr(out, C.c_double), out.size)
        return [{"weight": out[3 * s], "macroparticles": out[3 * s + 1], "weight_v2": out[3 * s + 2]}
                for s in range(self.nspecies)]

    def set_denoiser(self, dn, enabled: bool = True):
        """rhgpu_set_denoiser: apply `dn` to the moments in every step (None: none)."""
        self.lib.call("set_denoiser", self.h, dn.h if dn is not None else None, 1 if enabled else 0)

    def set_path(self, path: int):
        self.lib.call("set_path", self.h, path)

    def select_path(self, fast: bool):
        """The B200 library's particle path, or the oracle's matching order:
        fast = dual-cell storage order, else the reference's order."""
        if self.lib.has("set_path"):
            self.set_path(PATH_FAST if fast else PATH_EXACT)
        elif self.lib.has("set_deposit_order"):
            self.set_deposit_order(1 if fast else 0)
        elif fast:
            raise RuntimeError(f"{self.lib.prefix}: no fast-path order")

    def set_threads(self, n: int):
        self.lib.call("set_threads", self.h, n)


_GPU_LIB: Optional[Library] = None


def philox4x32(lib: "Library", ctr, key) -> list:
    """The library's Philox-4x32-10 (host side) of a 4-word counter and 2-word key."""
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib.fn["philox4x32"](c, k, o)
    return list(o)


def neutral_density(lib: "Library", injector, mass: float, xyz: np.ndarray, device: int = 0) -> np.ndarray:
    """rhgpu_neutral_density: an exosphere source's neutral density at points (n x 3, metres)."""
    p = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    out = np.empty(p.shape[0], dtype=np.float64)
    lib.call("neutral_density", C.cast(C.byref(injector), C.c_void_p), mass, p.shape[0], _ptr(p, C.c_double),
             _ptr(out, C.c_double), device)
    return out


def gpu_library_path() -> str:
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "librhgpu.so")


def gpu_library() -> Library:
    """Loads the B200 library; raises if it has not been built. There is no
    fallback: without the CUDA library the package cannot run the hot path."""
    global _GPU_LIB
    if _GPU_LIB is None:
        path = gpu_library_path()
        if not os.path.exists(path):
            raise RuntimeError(f"rhybrid_b200: CUDA library {path} not built (run __graft_entry__.build())")
        _GPU_LIB = Library(path, "rhgpu_")
    return _GPU_LIB


class Denoiser:
    """rhgpu_dn: the learned moment denoiser (BF16 tensor-core network)."""

    def __init__(self, lib: Library, nx: int, ny: int, nz: int, periodic, pair_capacity: int = 0, device: int = 0):
        self.lib = lib
        self.ncells = nx * ny * nz
        per = (C.c_int32 * 3)(*[1 if p else 0 for p in periodic])
        h = C.c_void_p()
        lib.call("dn_create", nx, ny, nz, per, pair_capacity, device, C.byref(h))
        self.h = h

    def close(self):
        if self.h:
            self.lib.call("dn_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, p: np.ndarray):
        a = np.ascontiguousarray(p, dtype=np.float32)
        assert a.size == DN_PARAMS
        self.lib.call("dn_set_params", self.h, _ptr(a, C.c_float), a.size)

    def params(self) -> np.ndarray:
        a = np.zeros(DN_PARAMS, dtype=np.float32)
        self.lib.call("dn_get_params", self.h, _ptr(a, C.c_float), a.size)
        return a

    def set_scales(self, rho_scale: float, j_scale: float):
        self.lib.call("dn_set_scales", self.h, rho_scale, j_scale)

    def set_velocity_form(self, enabled: bool):
        """rhgpu_dn_set_velocity_form: the network sees rho and J/rho (j_scale a
        speed) and hands back J = rho' u'."""
        self.lib.call("dn_set_velocity_form", self.h, 1 if enabled else 0)

    def set_keep_mask(self, keep):
        """rhgpu_dn_set_keep_mask: cells (nonzero) whose moments the network
        leaves as deposited; None clears it."""
        if keep is None:
            self.lib.call("dn_set_keep_mask", self.h, None)
            return
        k = np.ascontiguousarray(keep, dtype=np.uint8).reshape(-1)
        if k.size != self.ncells:
            raise ValueError(f"keep mask of {k.size} cells for {self.ncells}")
        self.lib.call("dn_set_keep_mask", self.h, k.ctypes.data_as(C.c_void_p))

    def apply(self, rho: np.ndarray, ji: np.ndarray, min_rho: float = -np.inf):
        r = np.ascontiguousarray(rho, dtype=np.float64).reshape(-1)
        j = np.ascontiguousarray(ji, dtype=np.float64).reshape(-1)
        ro, jo = np.empty_like(r), np.empty_like(j)
        self.lib.call("dn_apply", self.h, _ptr(r, C.c_double), _ptr(j, C.c_double), _ptr(ro, C.c_double),
                      _ptr(jo, C.c_double), min_rho)
        return ro, jo.reshape(-1, 3)

    def loss_grad(self, rho, ji, rho_t, ji_t):
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (rho, ji, rho_t, ji_t)]
        loss = C.c_double()
        g = np.zeros(DN_PARAMS, dtype=np.float32)
        self.lib.call("dn_loss_grad", self.h, *[_ptr(a, C.c_double) for a in arrs], C.byref(loss), _ptr(g, C.c_float))
        return loss.value, g

    def add_pair(self, ctx, factor: int, offset: int):
        self.lib.call("dn_add_pair", self.h, ctx.h, factor, offset)

    def add_crops(self, ctx, factor: int, offset: int, origins):
        """rhgpu_dn_add_crops: one pair per crop of ctx's grid; origins (n x 3) cell
        indices of the crops' corners, the crop size being this denoiser's grid."""
        o = np.ascontiguousarray(origins, dtype=np.int32).reshape(-1, 3)
        self.lib.call("dn_add_crops", self.h, ctx.h, factor, offset, o.shape[0], o.ctypes.data_as(C.c_void_p))

    def set_loss_border(self, border: int):
        self.lib.call("dn_set_loss_border", self.h, border)

    def train(self, iterations: int, lr: float) -> float:
        loss = C.c_double()
        self.lib.call("dn_train", self.h, iterations, lr, C.byref(loss))
        return loss.value

    def pair_error(self, pair: int):
        out = np.zeros(4)
        self.lib.call("dn_pair_error", self.h, pair, _ptr(out, C.c_double))
        return {"raw_rho": out[0], "raw_J": out[1], "dn_rho": out[2], "dn_J": out[3]}

    def num_pairs(self):
        n, newest = C.c_int32(), C.c_int32()
        self.lib.call("dn_num_pairs", self.h, C.byref(n), C.byref(newest))
        return n.value, newest.value
