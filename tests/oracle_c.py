"""ctypes wrapper of the C restatement oracle (oracle/_build/liboracle.so,
built by `make -C oracle oracle`).  Test infrastructure."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "oracle" / "_build" / "liboracle.so"


class System(C.Structure):
    _fields_ = [("n", C.c_int * 3), ("cells", C.c_int * 3), ("L", C.c_double * 3), ("dt", C.c_double),
                ("gravity", C.c_double), ("flow_dir", C.c_int), ("wall_s", C.c_double),
                ("sqrt_t_over_m", C.c_double), ("vox", C.c_void_p), ("nrm", C.c_void_p), ("t1", C.c_void_p),
                ("t2", C.c_void_p), ("seed", C.c_uint64), ("wall_model", C.c_int), ("alpha_n", C.c_double),
                ("alpha_t", C.c_double), ("cl_vmax", C.c_double)]


class Gas(C.Structure):
    _fields_ = [("mass", C.c_double), ("diam", C.c_double), ("density", C.c_double),
                ("atoms_per_molecule", C.c_double), ("volume_global", C.c_double)]


class Counters(C.Structure):
    _fields_ = [("count_periodic", C.c_longlong * 3), ("wall_hits", C.c_ulonglong), ("reseeds", C.c_ulonglong),
                ("collisions", C.c_ulonglong), ("candidates", C.c_ulonglong)]


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


T0 = 1.65088e-21 / 1.3806503e-23   # temperature unit (dsmc/unitconverter.cpp)
NUMBER_DENSITY0 = 1.0 / (1e-6 * 1e-6 * 1e-6)   # 1 / L0^3, m^-3 (dsmc/unitconverter.cpp:20)


class Oracle:
    """One system of the C oracle: geometry arrays, gas settings and state."""

    def __init__(self, geometry, settings: dict, seed: int):
        self.lib = C.CDLL(str(LIB))
        L = self.lib
        L.oracle_init.argtypes = [C.POINTER(System), C.c_long, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.oracle_accelerate.argtypes = [C.POINTER(System), C.c_long, C.POINTER(C.c_double)]
        L.oracle_move.argtypes = [C.POINTER(System), C.c_long, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                  C.c_uint32, C.POINTER(Counters)]
        L.oracle_cells_layout.argtypes = [C.POINTER(System), C.c_double, C.c_double] + [C.c_void_p] * 6
        L.oracle_cells_layout.restype = C.c_int
        L.oracle_sort.argtypes = [C.POINTER(System), C.c_long, C.POINTER(C.c_double)] + [C.c_void_p] + [C.c_int] + \
            [C.c_void_p] * 4
        L.oracle_sort.restype = C.c_int
        L.oracle_collide.argtypes = [C.POINTER(System), C.c_int] + [C.c_void_p] * 8 + [C.c_uint32,
                                                                                       C.POINTER(Counters)]
        L.oracle_sample_profiles.argtypes = [C.POINTER(System), C.c_long, C.POINTER(C.c_double),
                                             C.POINTER(C.c_double), C.c_double, C.c_double, C.c_int,
                                             C.POINTER(C.c_double)]
        L.oracle_measures.argtypes = [C.POINTER(System), C.POINTER(Gas), C.c_long, C.POINTER(C.c_double),
                                      C.c_longlong, C.c_double, C.POINTER(C.c_double)]
        self.g = geometry
        st = settings
        self.vox = np.ascontiguousarray(geometry.voxels)
        self.nrm = np.ascontiguousarray(geometry.normals)
        self.t1 = np.ascontiguousarray(geometry.tangents1)
        self.t2 = np.ascontiguousarray(geometry.tangents2)
        s = System()
        s.n[:] = list(geometry.shape)
        s.cells[:] = [st["cells_x"], st["cells_y"], st["cells_z"]]
        s.L[:] = [st["Lx"], st["Ly"], st["Lz"]]
        s.dt = st["dt"]
        s.gravity = st["gravity"]
        s.flow_dir = st["flow_direction"]
        s.wall_s = float(np.sqrt(st["wall_temperature"] / T0 / st["mass"]))
        s.sqrt_t_over_m = float(np.sqrt(st["temperature"] / T0 / st["mass"]))
        s.vox = self.vox.ctypes.data
        s.nrm = self.nrm.ctypes.data
        s.t1 = self.t1.ctypes.data
        s.t2 = self.t2.ctypes.data
        s.seed = seed
        s.wall_model = {"thermal": 0, "specular": 1, "cercignani_lampis": 2}[st.get("surface", "thermal")]
        s.alpha_n = st.get("alpha_n", 0.5)
        s.alpha_t = st.get("alpha_t", 0.8)
        L0, m0, E0 = 1e-6, 1.66053886e-27, 1.65088e-21   # dsmc/unitconverter.cpp:3-21
        s.cl_vmax = 1500.0 / (L0 / (L0 * np.sqrt(m0 / E0)))
        self.s = s
        ncell = int(np.prod(s.cells[:]))
        self.cell_map = np.empty(ncell, np.int32)
        nc = L.oracle_cells_layout(C.byref(s), st["atoms_per_molecule"], st["diam"], None, None, None, None, None, None)
        self.global_index = np.empty(nc, np.int32)
        self.coeff = np.empty(nc)
        self.volume = np.empty(nc)
        L.oracle_cells_layout(C.byref(s), st["atoms_per_molecule"], st["diam"], self.cell_map.ctypes.data,
                              self.global_index.ctypes.data, None, None, self.volume.ctypes.data,
                              self.coeff.ctypes.data)
        self.num_cells = nc
        self.vr_max = np.full(nc, 3 * np.sqrt(st["temperature"] / T0))
        self.rest = np.zeros(nc)
        self.c = Counters()
        self.r = np.zeros((0, 3))
        self.v = np.zeros((0, 3))
        # the sampler (StatisticsSampler, dsmc/statisticssampler.cpp:13-42)
        self.mass = st["mass"]
        self.temperature = st["temperature"] / T0
        self.bins = st.get("sampling_bins", 1)
        self.prof_sums = np.zeros(4 * self.bins)
        self.t = 0.0
        self.gas = Gas(mass=st["mass"], diam=st["diam"], density=st.get("density", 0.0) / NUMBER_DENSITY0,
                       atoms_per_molecule=st["atoms_per_molecule"], volume_global=0.0)

    def init(self, n: int):
        self.r = np.zeros((n, 3))
        self.v = np.zeros((n, 3))
        self.lib.oracle_init(C.byref(self.s), n, _p(self.r), _p(self.v))

    def set(self, r, v):
        self.r = np.array(r, np.float64, copy=True, order="C")
        self.v = np.array(v, np.float64, copy=True, order="C")

    def move(self, step: int):
        n = len(self.r)
        self.lib.oracle_accelerate(C.byref(self.s), n, _p(self.v))
        self.lib.oracle_move(C.byref(self.s), n, _p(self.r), _p(self.v), step, C.byref(self.c))

    def sort(self):
        n = len(self.r)
        self.cell_of = np.empty(n, np.int32)
        self.count = np.empty(self.num_cells, np.int32)
        self.start = np.empty(self.num_cells, np.int32)
        self.members = np.empty(n, np.int32)
        rc = self.lib.oracle_sort(C.byref(self.s), n, _p(self.r), self.cell_map.ctypes.data, self.num_cells,
                                  self.cell_of.ctypes.data, self.count.ctypes.data, self.start.ctypes.data,
                                  self.members.ctypes.data)
        assert rc == 0, "particle in a cell with no free volume"

    def collide(self, step: int):
        self.lib.oracle_collide(C.byref(self.s), self.num_cells, self.global_index.ctypes.data,
                                self.coeff.ctypes.data, self.vr_max.ctypes.data, self.rest.ctypes.data,
                                self.count.ctypes.data, self.start.ctypes.data, self.members.ctypes.data,
                                self.v.ctypes.data, step, C.byref(self.c))

    def step(self, step: int):
        self.move(step)
        self.sort()
        self.collide(step)
        self.t += self.s.dt  # System::step (dsmc/system.cpp:24-26)

    def sample(self):
        """StatisticsSampler::sample's profiles after a step (every step
        sampled): adds into prof_sums."""
        self.lib.oracle_sample_profiles(C.byref(self.s), len(self.r), _p(self.r), _p(self.v), self.mass,
                                        self.temperature, self.bins, _p(self.prof_sums))

    def profile_sums(self) -> np.ndarray:
        """(4, bins): count, sum v_z and sum 1/2 m v_z^2 per y bin, then the
        v_x histogram (the layout of the reference harness's sums)."""
        p = self.prof_sums
        return np.stack([p[0:3 * self.bins:3], p[1:3 * self.bins:3], p[2:3 * self.bins:3], p[3 * self.bins:]])

    def measures(self, volume_global: float) -> np.ndarray:
        """energy (eV), temperature (K), number and volumetric flow rate,
        pressure (Pa), permeability (darcy) of the current state."""
        self.gas.volume_global = volume_global
        out = np.zeros(6)
        fd = self.s.flow_dir
        self.lib.oracle_measures(C.byref(self.s), C.byref(self.gas), len(self.v), _p(self.v),
                                 self.c.count_periodic[fd], self.t, _p(out))
        return out

    @property
    def cell_global_of_particles(self):
        return self.global_index[self.cell_of]

    def counters(self):
        return {"count_periodic": list(self.c.count_periodic), "wall_collisions": self.c.wall_hits,
                "collisions": self.c.collisions, "reseeds": self.c.reseeds}
