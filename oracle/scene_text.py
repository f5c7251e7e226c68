"""CPU ORACLE - test infrastructure only: scene, configuration and task files.

A Python restatement of the reference's readers, used by the tests as an
independent check of the product's C++ readers and to feed the C++ oracle:

  * SceneLoader::SceneFileRead      Scene/SceneLoader.cpp:243-353 (+ checkScene :200-238)
  * scene grammar D(R(GH+)+)+       Tool/FileLoader/RegularExpressionTree.cpp:47-71
  * SceneConfiguration::loadConfiguration  Scene/SceneConfiguration.cpp:39-69
  * TaskLoader::loadRayTracingHeliostatIndex  RayTracingPipeline/TaskLoader.cpp:114-204

Numbers are converted as the reference converts them: `istream >> float`
rounds the decimal text straight to float (glibc strtof, called here through
ctypes); JSON numbers become doubles first and are then narrowed to float,
as nlohmann::json does.
"""
from __future__ import annotations

import ctypes
import json
from dataclasses import dataclass, field

import numpy as np

_libc = ctypes.CDLL(None)
_libc.strtof.restype = ctypes.c_float
_libc.strtof.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p)]
_libc.strtol.restype = ctypes.c_long
_libc.strtol.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int]


class SceneError(Exception):
    """The reference prints the message and returns false."""


class _Stream:
    """Whitespace tokens with line-rest skipping, like std::istream >> / getline."""

    def __init__(self, text: str):
        self.s = text
        self.i = 0
        self.failed = False

    def token(self) -> str | None:
        s, n = self.s, len(self.s)
        i = self.i
        while i < n and s[i] in " \t\n\r\v\f":
            i += 1
        if i >= n:
            self.i = i
            self.failed = True
            return None
        j = i
        while j < n and s[j] not in " \t\n\r\v\f":
            j += 1
        self.i = j
        return s[i:j]

    def rest_of_line(self) -> None:
        k = self.s.find("\n", self.i)
        self.i = len(self.s) if k < 0 else k + 1

    def f32(self) -> np.float32:
        if self.failed:
            return np.float32(0.0)
        t = self.token()
        if t is None:
            return np.float32(0.0)
        b = t.encode()
        end = ctypes.c_char_p()
        v = _libc.strtof(b, ctypes.byref(end))
        if ctypes.cast(end, ctypes.c_void_p).value == ctypes.cast(ctypes.c_char_p(b), ctypes.c_void_p).value:
            self.failed = True
            return np.float32(0.0)
        return np.float32(v)

    def i32(self) -> int:
        if self.failed:
            return 0
        t = self.token()
        if t is None:
            return 0
        try:
            return int(t)
        except ValueError:
            # istream >> int reads a leading integer prefix
            k = 0
            if k < len(t) and t[k] in "+-":
                k += 1
            while k < len(t) and t[k].isdigit():
                k += 1
            if k == 0 or (k == 1 and t[0] in "+-"):
                self.failed = True
                return 0
            return int(t[:k])


@dataclass
class Receiver:
    type: int
    pos: np.ndarray
    size: np.ndarray
    norm: np.ndarray
    face: int


@dataclass
class Grid:
    type: int
    receiver: int
    start: int
    pos: np.ndarray
    size: np.ndarray
    inter: np.ndarray
    n: int
    helio_type: int


@dataclass
class Heliostat:
    type: int
    grid: int
    pos: np.ndarray
    size: np.ndarray
    gap: np.ndarray
    matrix: tuple
    surface: np.ndarray
    local_centers: list = field(default_factory=list)
    local_normals: list = field(default_factory=list)


@dataclass
class SceneText:
    ground: tuple
    grid_num: int
    receivers: list
    grids: list
    heliostats: list


_NEXT = {"start": {"D": "ground"}, "ground": {"R": "recv"}, "recv": {"G": "grid"}, "grid": {"H": "helio"},
         "helio": {"R": "recv", "G": "grid", "H": "helio"}}


def _step(state: str, c: str) -> str:
    nxt = _NEXT[state].get(c)
    if nxt is None:
        raise SceneError("Cannot step forward.")
    return nxt


def _key(st: _Stream, name: str) -> None:
    if st.token() != name:
        raise SceneError(f"Miss ' {name} ' property.")


def _vec(st: _Stream, name: str) -> np.ndarray:
    _key(st, name)
    return np.array([st.f32(), st.f32(), st.f32()], dtype=np.float32)


def parse_scene(text: str) -> SceneText:
    """SceneLoader::SceneFileRead; raises SceneError where it returns false."""
    matrix = (1, 1)
    gap = np.zeros(2, np.float32)
    surface = np.full(6, -1.0, np.float32)
    centers: list = []
    normals: list = []
    n_centers = n_normals = 0
    recv_id = -1
    total = 0
    helio_type = -1
    state = "start"
    ground = (np.float32(0), np.float32(0))
    grid_num = 0
    receivers, grids, helios = [], [], []
    st = _Stream(text)
    while True:
        head = st.token()
        if head is None:
            break
        if head[0] == "#":
            st.rest_of_line()
            continue
        if head == "gap":
            gap = np.array([st.f32(), st.f32()], np.float32)
        elif head == "matrix":
            matrix = (st.i32(), st.i32())
        elif head == "surface_property":
            surface = np.array([st.f32() for _ in range(6)], np.float32)
        elif head == "ground":
            state = _step(state, "D")
            ground = (st.f32(), st.f32())
            _key(st, "ngrid")
            grid_num = st.i32()
        elif head == "Recv":
            state = _step(state, "R")
            t = st.i32()
            if t not in (0, 1):
                raise SceneError("Receiver type has not defined.")
            pos, size, norm = _vec(st, "pos"), _vec(st, "size"), _vec(st, "norm")
            _key(st, "face")
            face = st.i32()
            _key(st, "end")
            receivers.append(Receiver(t, pos, size, norm, face))
            recv_id += 1
        elif head == "Grid":
            state = _step(state, "G")
            t = st.i32()
            if t != 0:
                raise SceneError("Grid type has not defined.")
            pos, size, inter = _vec(st, "pos"), _vec(st, "size"), _vec(st, "inter")
            _key(st, "n")
            n = st.i32()
            _key(st, "type")
            helio_type = st.i32()
            _key(st, "end")
            grids.append(Grid(t, recv_id, total, pos, size, inter, n, helio_type))
        elif head == "helio":
            state = _step(state, "H")
            if helio_type not in (0, 1):
                raise SceneError("Heliostat has not defined.")
            pos = np.array([st.f32() for _ in range(3)], np.float32)
            size = np.array([st.f32() for _ in range(3)], np.float32)
            h = Heliostat(helio_type, len(grids) - 1, pos, size, gap.copy(), matrix, surface.copy())
            if int(surface[1]) == 1:
                h.local_centers = list(centers)
                h.local_normals = list(normals)
            helios.append(h)
            centers, normals = [], []
            n_centers = n_normals = 0
            total += 1
        elif head == "subhelio":
            st.rest_of_line()
            while n_centers < matrix[0] * matrix[1]:
                centers.append(np.array([st.f32(), st.f32(), st.f32()], np.float32))
                st.rest_of_line()
                n_centers += 1
            while n_normals < matrix[0] * matrix[1]:
                normals.append(np.array([st.f32(), st.f32(), st.f32()], np.float32))
                st.rest_of_line()
                n_normals += 1
        else:
            state = _step(state, "?")
    # checkScene
    if grid_num != len(grids):
        raise SceneError(f"The scene should contains {grid_num} grids, but got {len(grids)} grids.")
    for i, g in enumerate(grids):
        exist = (len(helios) if i == len(grids) - 1 else grids[i + 1].start) - g.start
        if exist != g.n:
            raise SceneError(f"grid {i + 1} should contain {g.n} heliostat(s), but got {exist}")
        if i == 0 and g.receiver != 0:
            raise SceneError("the first grid must belong to receiver 0")
        if i > 0 and g.receiver not in (grids[i - 1].receiver, grids[i - 1].receiver + 1):
            raise SceneError("grid receiver index out of order")
    return SceneText(ground, grid_num, receivers, grids, helios)


CONFIG_DEFAULTS = {
    "sun_dir": [1.0, 0.0, 0.0], "dni": 1000.0, "csr": 0.1, "num_of_sunshape_groups": 128,
    "num_per_sunshape_group": 2048, "inverse_transform_sampling_groups": 1024, "receiver_pixel_length": 0.01,
    "helio_disturb_std": 0.001, "helio_pixel_length": 0.01, "helio_reflected_rate": 0.88,
}
_INT_KEYS = {"num_of_sunshape_groups", "num_per_sunshape_group", "inverse_transform_sampling_groups"}


def parse_config(text: str) -> tuple[dict, int]:
    """SceneConfiguration::loadConfiguration: (values, number of keys set)."""
    data = json.loads(text)
    if not isinstance(data, dict):
        raise ValueError("configuration must be a JSON object")
    out = {}
    n = 0
    for key, default in CONFIG_DEFAULTS.items():
        if key in data:
            n += 1
            v = data[key]
            if key == "sun_dir":
                out[key] = np.array([np.float32(float(x)) for x in v[:3]], np.float32)
            elif key in _INT_KEYS:
                out[key] = int(v)
            else:
                out[key] = np.float32(float(v))
        else:
            if key == "sun_dir":
                out[key] = np.array(default, np.float32)
            elif key in _INT_KEYS:
                out[key] = int(default)
            else:
                out[key] = np.float32(default)
    return out, n


def parse_tasks(text: str, num_heliostats: int, grid_of) -> tuple[list, list, bool]:
    """TaskLoader::loadRayTracingHeliostatIndex: (heliostats, grid ids, status);
    raises ValueError where the reference throws."""
    st = _Stream(text)
    tok = st.token() or ""
    try:
        n = int(tok)
    except ValueError:
        raise ValueError(f"The number of heliostats '{tok}' is invalid.")
    if n <= 0:
        raise ValueError(f"The number of heliostats '{tok}' is invalid.")
    helios, recvs, ok = [], [], True
    prev = tok
    for i in range(n):
        if st.i >= len(st.s):
            raise ValueError(f"{n} heliostat(s) are expected. But only got {i} heliostats.")
        t = st.token()
        if t is None:
            t = prev  # a failed extraction leaves the previous token in place
        prev = t
        try:
            hid = int(t)
        except ValueError:
            raise ValueError(f"The {i + 1}-th heliostat index '{t}' is invalid.")
        if hid < 0 or hid >= num_heliostats:
            raise ValueError(f"The {i + 1}-th heliostat index '{t}' is invalid.")
        if hid not in helios:
            helios.append(hid)
            g = grid_of(hid)
            if g not in recvs:
                recvs.append(g)
        else:
            ok = False
    if st.token() is not None:
        return helios, recvs, False
    return helios, recvs, ok
