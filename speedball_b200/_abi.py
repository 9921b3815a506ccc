"""ctypes binding of libspeedball_cuda.so (include/speedball_cuda.h, speedball_scene.h).

The library is loaded from this package directory; there is no fallback:
a missing library raises ``LibraryMissing`` and every device call goes
through the CUDA path.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
# SB_LIB_PATH selects another build of the same library (e.g. a tuning variant)
LIB_PATH = Path(os.environ.get("SB_LIB_PATH", HERE / "libspeedball_cuda.so"))

SB_OK = 0
STATUS_NAMES = {
    0: "SB_OK", 1: "SB_ERR_INVALID_ARG", 2: "SB_ERR_LAYOUT_VIOLATION", 3: "SB_ERR_OOM",
    4: "SB_ERR_CUDA", 5: "SB_ERR_DEVICE_WATCHDOG", 6: "SB_ERR_UNSUPPORTED",
    7: "SB_ERR_NO_DEVICE", 8: "SB_ERR_NOT_READY",
}
SB_ERR_INVALID_ARG, SB_ERR_LAYOUT_VIOLATION, SB_ERR_OOM = 1, 2, 3
SB_ERR_CUDA, SB_ERR_DEVICE_WATCHDOG, SB_ERR_UNSUPPORTED = 4, 5, 6
SB_ERR_NO_DEVICE, SB_ERR_NOT_READY = 7, 8

SB_CTX_RECORD_HITS = 1

BUF = dict(
    BVH_NODES=0, TRI_INDEX=1, VERTEX_DATA=2, TRI_MATERIAL=3, MATERIALS=4, LIGHTS=5,
    IRRADIANCE_HISTORY=6, DEPTH_HISTORY=7, IRRADIANCE_ATLAS=8, DEPTH_ATLAS=9, RAY_DATA=10,
    HIT_RECORDS=11, VISIBILITY=12, TLAS_ORDER=13, INSTANCE_BOUNDS=14, RECORD_E=15, EMITTER_VIS=16,
    ROUGH_SPECULAR=17, ROUGH_ATLAS=18, GLOSSY_SPECULAR=19, GLOSSY_WEIGHT=20, GLOSSY_ATLAS=21,
)


class LibraryMissing(RuntimeError):
    """libspeedball_cuda.so is not built; run speedball_b200/build.py."""


class SbError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class sb_device_opts(C.Structure):
    _fields_ = [("device", C.c_int32), ("flags", C.c_uint32)]


class sb_scene_view(C.Structure):
    _fields_ = [
        ("bvhNodes", C.c_void_p), ("nodeCount", C.c_uint32),
        ("triIndex", C.c_void_p), ("triCount", C.c_uint32),
        ("vertexData", C.c_void_p), ("vertexCount", C.c_uint32),
        ("triMaterial", C.c_void_p),
        ("materials", C.c_void_p), ("materialsLen", C.c_uint32),
        ("materialCount", C.c_uint32), ("instBase", C.c_uint32), ("instCount", C.c_uint32),
        ("tlasBase", C.c_uint32), ("tlasNodeCount", C.c_uint32),
    ]


class sb_grid(C.Structure):
    _fields_ = [
        ("gridMin", C.c_float * 3), ("gridSize", C.c_float * 3), ("res", C.c_uint32 * 3),
        ("raysPerProbe", C.c_uint32), ("maxDist", C.c_float), ("cellMin", C.c_float),
    ]


# Field order of sb_params (and of the oracle's Params) — gi_probes.js:1198-1255.
PARAM_NAMES = [
    "frameJitter", "emitterVisSeed", "hysteresis", "hysteresisExponent",
    "depthSharpness", "radianceClamp", "classifyStrength", "filterStrength", "filterSmooth",
    "tempChangeSigma1", "tempChangeHDrop", "tempClampSigma", "nirGate", "nirGain", "skyIntensity",
] + [f"skySH{i}" for i in range(27)] + [
    "debugTraceBiasScale", "debugRayEpsScale", "debugDirectScale", "debugEmissiveScale",
    "debugAlbedoScale", "debugBounceScale", "debugCosinePower",
    "debugTempNoiseHBoost", "debugTempChangeSigma0", "debugTempMinChangeH",
    "debugTempVarEps", "debugTempVarRel", "debugDepthHistoryScale",
    "debugFilterKScale", "debugFilterRelScale", "debugFilterEpsScale",
    "reflectionSkyFallback", "skyConfigured",
]


class sb_params(C.Structure):
    _fields_ = [(n, C.c_float) for n in PARAM_NAMES[:15]] + [("skySH", C.c_float * 27)] + [
        (n, C.c_float) for n in PARAM_NAMES[42:]
    ]

    def to_array(self) -> np.ndarray:
        """All fields in declaration order (the oracle's parameter vector)."""
        out = []
        for n in PARAM_NAMES:
            out.append(self.skySH[int(n[5:])] if n.startswith("skySH") else getattr(self, n))
        return np.array(out, dtype=np.float64)


class sb_solve_item(C.Structure):
    _fields_ = [("ctx", C.c_void_p), ("cascade", C.c_uint32), ("probeOffset", C.c_uint32),
                ("updatedCount", C.c_uint32)]


class sb_frame_lane(C.Structure):
    _fields_ = [("ctx", C.c_void_p), ("refitRoots", C.c_void_p), ("refitEnds", C.c_void_p),
                ("refitCount", C.c_uint32), ("refitTlas", C.c_int32)]


class sb_grads(C.Structure):
    _fields_ = [("dAlbedo", C.c_void_p), ("dEmissive", C.c_void_p), ("dIntensity", C.c_void_p)]


class sb_tuning(C.Structure):
    _fields_ = [("traceBlock", C.c_uint32), ("sortKey", C.c_uint32), ("smemTlasNodes", C.c_uint32),
                ("bvhKind", C.c_uint32), ("smemWideNodes", C.c_uint32)]


REFLECT_TIERS = {"off": 0, "rough": 1, "high": 2, "ultra": 3}


class sb_reflection_layout(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("tier", "glossyOct", "glossyTile", "glossyInterval", "glossyTilesX",
                                          "glossyTilesY", "glossyAtlasW", "glossyAtlasH", "glossyPhase")]


class sb_gather_params(C.Structure):
    _fields_ = [("normalBias", C.c_float * 2), ("chebyBias", C.c_float * 2), ("chebyStrength", C.c_float),
                ("detailStrength", C.c_float), ("intensity", C.c_float), ("enabled", C.c_float),
                ("samplePositionScale", C.c_float), ("sampleBiasScale", C.c_float), ("borderBand", C.c_float),
                ("cascades", C.c_uint32), ("dualDetail", C.c_uint32), ("reflectionIntensity", C.c_float),
                ("roughnessLimit", C.c_float)]


class sb_stats(C.Structure):
    _fields_ = [("primaryRays", C.c_uint64), ("shadowRays", C.c_uint64),
                ("tlasNodeVisits", C.c_uint64), ("instanceVisits", C.c_uint64),
                ("blasNodeVisits", C.c_uint64), ("triangleTests", C.c_uint64),
                ("lastSolveMs", C.c_float), ("lastTraceMs", C.c_float), ("lastBlendMs", C.c_float),
                ("kernelLaunches", C.c_uint64), ("lastPrimaryMs", C.c_float), ("lastShadowMs", C.c_float),
                ("lastShadeMs", C.c_float), ("shadowTlasNodeVisits", C.c_uint64),
                ("shadowInstanceVisits", C.c_uint64), ("shadowBlasNodeVisits", C.c_uint64),
                ("shadowTriangleTests", C.c_uint64), ("lastForwardRecordMs", C.c_float),
                ("lastBackwardMs", C.c_float), ("sceneBvhBuilds", C.c_uint64), ("sceneBvhActive", C.c_uint32),
                ("lastSceneBvhBuildMs", C.c_float), ("lastEmitMs", C.c_float),
                ("sceneBvhBuilding", C.c_uint32)]


_P = C.c_void_p
_U32 = C.c_uint32
# name -> (restype, argtypes)
SIGNATURES = {
    "sb_create": (C.c_int, [C.POINTER(sb_device_opts), C.POINTER(C.c_void_p)]),
    "sb_destroy": (None, [_P]),
    "sb_last_error": (C.c_char_p, [_P]),
    "sb_abi_version": (_U32, []),
    "sb_set_stream": (C.c_int, [_P, _P]),
    "sb_set_walk_step_limit": (C.c_int, [_P, C.c_uint32]),
    "sb_triangle_test": (C.c_uint32, []),
    "sb_fit_fine_box": (C.c_int, [_P, _P, _P, _P, _P, _P]),
    "sb_set_reflection_quality": (C.c_int, [_P, _U32]),
    "sb_get_reflection_layout": (C.c_int, [_P, _U32, C.POINTER(sb_reflection_layout)]),
    "sb_rebuild_scene_bvh": (C.c_int, [_P]),
    "sb_set_scene_bvh_build_mode": (C.c_int, [_P, _U32]),
    "sb_finish_scene_bvh": (C.c_int, [_P]),
    "sb_build_blas_device": (C.c_int, [_P, _P, C.c_uint32, _P, C.c_uint32, C.c_uint32, _P, _P, _P]),
    "sb_build_blas_gpu": (C.c_int, [_P, _P, C.c_uint32, _P, C.c_uint32, C.c_uint32, _P, _P, _P]),
    "sb_probe_rays": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint32, _P, _P]),
    "sb_gather_params_defaults": (None, [_P]),
    "sb_gather_irradiance": (C.c_int, [_P, _P, _P, _P, _P, C.c_uint32, _P]),
    "sb_gather_reflections": (C.c_int, [_P, _P, _P, _P, _P, _P, C.c_uint32, _P, _P]),
    "sb_raycast_device": (C.c_int, [_P, _P, _P, C.c_uint32, _P, _P, _P]),
    "sb_occluded_device": (C.c_int, [_P, _P, _P, _P, C.c_uint32, _P]),
    "sb_synchronize": (C.c_int, [_P]),
    "sb_upload_scene": (C.c_int, [_P, C.POINTER(sb_scene_view)]),
    "sb_upload_range": (C.c_int, [_P, _U32, _U32, _U32, _P]),
    "sb_read_buffer": (C.c_int, [_P, _U32, _U32, _U32, _P]),
    "sb_read_buffer_async": (C.c_int, [_P, _U32, _U32, _U32, _P]),
    "sb_upload_lights": (C.c_int, [_P, _P, _U32, _U32, _U32, C.c_int32]),
    "sb_params_defaults": (None, [C.POINTER(sb_params)]),
    "sb_configure_cascade": (C.c_int, [_P, _U32, C.POINTER(sb_grid)]),
    "sb_set_params": (C.c_int, [_P, C.POINTER(sb_params)]),
    "sb_solve": (C.c_int, [_P, _U32, _U32, _U32]),
    "sb_solve_batch": (C.c_int, [C.POINTER(sb_solve_item), _U32]),
    "sb_raycast": (C.c_int, [_P, _P, _P, _U32, _P, _P, _P]),
    "sb_occluded": (C.c_int, [_P, _P, _P, _P, _U32, _P]),
    "sb_refit_blas": (C.c_int, [_P, _U32, _U32]),
    "sb_refit_blas_static": (C.c_int, [_P, _U32, _P, _U32, _P, _U32, _U32, _U32, _P, C.c_char_p, C.c_size_t]),
    "sb_update_deform": (C.c_int, [_P, _U32, _U32, _P, _U32, _U32]),
    "sb_update_deform_xyz": (C.c_int, [_P, _U32, _U32, _P, _P, _U32, _U32]),
    "sb_set_instances": (C.c_int, [_P, _U32, _P, _P, _P, _P]),
    "sb_build_tlas": (C.c_int, [_P]),
    "sb_update_transforms": (C.c_int, [_P, _P, _P, _U32]),
    "sb_forward_record": (C.c_int, [_P, _U32, _U32, _P, C.POINTER(C.c_double)]),
    "sb_backward": (C.c_int, [_P, C.POINTER(sb_grads)]),
    "sb_graph_capture_frame": (C.c_int, [_P, _U32, _U32, _U32, _P, _P, _U32, C.c_int32]),
    "sb_graph_launch": (C.c_int, [_P]),
    "sb_graph_capture_batch": (C.c_int, [C.POINTER(sb_frame_lane), _U32, C.POINTER(sb_solve_item), _U32]),
    "sb_graph_destroy": (C.c_int, [_P]),
    "sb_get_tuning": (C.c_int, [_P, C.POINTER(sb_tuning)]),
    "sb_set_tuning": (C.c_int, [_P, C.POINTER(sb_tuning)]),
    "sb_autotune": (C.c_int, [_P, _U32, C.POINTER(sb_tuning)]),
    "sb_autotune_batch": (C.c_int, [C.POINTER(sb_solve_item), _U32, C.POINTER(sb_tuning)]),
    "sb_get_stats": (C.c_int, [_P, C.POINTER(sb_stats)]),
    "sb_enable_counters": (C.c_int, [_P, C.c_int32]),
    "sbh_build_blas": (_U32, [_P, _U32, _P, _U32, _U32, _P, _P]),
    "sb_host_alloc": (C.c_int, [C.c_size_t, C.POINTER(C.c_void_p)]),
    "sb_host_free": (None, [_P]),
}


class PinnedArray:
    """A numpy view over page-locked host memory from sb_host_alloc."""

    def __init__(self, shape, dtype):
        self.dtype = np.dtype(dtype)
        n = int(np.prod(shape)) * self.dtype.itemsize
        p = C.c_void_p()
        check(load().sb_host_alloc(max(n, 1), C.byref(p)))
        self._p = p
        buf = (C.c_ubyte * max(n, 1)).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=self.dtype, count=int(np.prod(shape))).reshape(shape)

    def free(self):
        if self._p is not None and self._p.value:
            self.array = None
            load().sb_host_free(self._p)
            self._p = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

_lib = None


_variants: dict = {}


def load(variant: str | None = None) -> C.CDLL:
    """Load the library once; raise LibraryMissing when it is not built.
    `variant` names a build variant next to it, libspeedball_cuda_<variant>.so
    ("watertight": the watertight ray/triangle test)."""
    global _lib
    if variant is None and _lib is not None:
        return _lib
    if variant is not None and variant in _variants:
        return _variants[variant]
    path = LIB_PATH if variant is None else LIB_PATH.with_name(f"libspeedball_cuda_{variant}.so")
    if not path.exists():
        raise LibraryMissing(f"{path} is missing: build it with `python speedball_b200/build.py`")
    lib = C.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if variant is None:
        _lib = lib
    else:
        _variants[variant] = lib
    return lib


def ptr(a: np.ndarray | None) -> int | None:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays crossing the ABI must be C-contiguous"
    return a.ctypes.data


def check(status: int, ctx=None) -> None:
    if status != SB_OK:
        msg = load().sb_last_error(ctx).decode() if ctx else ""
        raise SbError(status, msg)


def default_params() -> sb_params:
    p = sb_params()
    load().sb_params_defaults(C.byref(p))
    return p
