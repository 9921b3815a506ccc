"""Autograd-style differentiation of the probe update (sb_forward_record /
sb_backward).

The reference has no adjoint; this is the host side of the library's own
forward/backward pair: the gradient of an irradiance-atlas loss with respect
to per-material albedo and emissive and per-light intensity, with hit records
and shadow visibility held at the ones the forward traced. Usage mirrors an
autograd function:

    adj = GIAdjoint(field, solves=2)
    loss = adj.forward(target)          # target: (probes, 36, 3) float32
    g = adj.backward()                  # dict of numpy arrays
    adj.setParameters(albedo=..., lightScale=...)

Light parameters are a scale s of each light record's colour (the record holds
colour x intensity, spectral_scene.js:724-813), so for a light of intensity I,
dL/dI = g["lightScale"] / I; `intensities` converts when given.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .field import ProbeField

MAT_STRIDE = 28
LIGHT_STRIDE = 17


class GIAdjoint:
    def __init__(self, field: ProbeField, solves: int = 2, cascade: int = 0):
        if not 1 <= solves <= 8:
            raise ValueError("solves must be in [1, 8]")
        self.field = field
        self.solves = solves
        self.cascade = cascade
        self._lib = field._lib
        mats = np.asarray(field._scene.materials, np.float32).reshape(-1, MAT_STRIDE)
        self.materialCount = mats.shape[0]
        self._albedo = mats[:, 0:3].astype(np.float64).copy()
        self._emissive = mats[:, 7:10].astype(np.float64).copy()
        recs = self._device_lights()
        self.lightCount = recs.shape[0]
        self._lightBase = recs[:, 7:10].copy()  # colour x intensity at scale 1
        self._lightScale = np.ones(self.lightCount)
        self._hasTarget = False
        r = field.getResolution()
        self.probes = int(r[0] * r[1] * r[2])

    def _device_lights(self) -> np.ndarray:
        n = self.field._lightCount
        out = np.zeros(n * LIGHT_STRIDE, np.float32)
        if n:
            self._ck(self._lib.sb_read_buffer(self.field.ctx, _abi.BUF["LIGHTS"], 0, out.size, _abi.ptr(out)))
        return out.reshape(n, LIGHT_STRIDE)

    def _ck(self, status):
        _abi.check(status, self.field.ctx)

    # ----------------------------------------------------------- parameters
    def parameters(self) -> dict:
        return dict(albedo=self._albedo.copy(), emissive=self._emissive.copy(), lightScale=self._lightScale.copy())

    def setParameters(self, albedo=None, emissive=None, lightScale=None) -> None:
        """Write changed values into the device records (colour fields only: the
        scene BVH and derived layouts stay valid)."""
        ctx = self.field.ctx
        for name, cur, off in (("albedo", albedo, 0), ("emissive", emissive, 7)):
            if cur is None:
                continue
            cur = np.asarray(cur, np.float64).reshape(self.materialCount, 3)
            old = self._albedo if name == "albedo" else self._emissive
            for m in np.nonzero((cur != old).any(axis=1))[0]:
                v = np.ascontiguousarray(cur[m], np.float32)
                self._ck(self._lib.sb_upload_range(ctx, _abi.BUF["MATERIALS"], int(m) * MAT_STRIDE + off, 3,
                                                   _abi.ptr(v)))
                old[m] = cur[m]
                self.field._scene.materials[m, off:off + 3] = v
        if lightScale is not None:
            s = np.asarray(lightScale, np.float64).reshape(self.lightCount)
            for l in np.nonzero(s != self._lightScale)[0]:
                v = np.ascontiguousarray(self._lightBase[l] * s[l], np.float32)
                self._ck(self._lib.sb_upload_range(ctx, _abi.BUF["LIGHTS"], int(l) * LIGHT_STRIDE + 7, 3,
                                                   _abi.ptr(v)))
                self._lightScale[l] = s[l]

    # -------------------------------------------------------- forward / backward
    def forward(self, target: np.ndarray | None = None):
        """`solves` feedback solves from a cleared history. Returns the loss
        sum (E - target)^2 over the last solve's interior irradiance texels when
        a target is given, else E itself as (probes, 36, 3) float32."""
        f = self.field
        self._ck(self._lib.sb_set_params(f.ctx, C.byref(f._params)))
        if target is None:
            self._ck(self._lib.sb_forward_record(f.ctx, self.cascade, self.solves, None, None))
            self._hasTarget = False
            return self.readE()
        t = np.ascontiguousarray(target, np.float32).reshape(-1)
        if t.size != self.probes * 36 * 3:
            raise ValueError(f"target has {t.size} values, expected {self.probes * 36 * 3}")
        loss = C.c_double(0.0)
        self._ck(self._lib.sb_forward_record(f.ctx, self.cascade, self.solves, _abi.ptr(t), C.byref(loss)))
        self._hasTarget = True
        return loss.value

    def readE(self) -> np.ndarray:
        e = np.zeros(self.probes * 36 * 4, np.float32)
        self._ck(self._lib.sb_read_buffer(self.field.ctx, _abi.BUF["RECORD_E"], 0, e.size, _abi.ptr(e)))
        return e.reshape(self.probes, 36, 4)[:, :, :3].copy()

    def backward(self, intensities: np.ndarray | None = None) -> dict:
        if not self._hasTarget:
            raise RuntimeError("backward needs a forward with a target")
        mc, lc = self.materialCount, self.lightCount
        ga = np.zeros(mc * 3, np.float32)
        ge = np.zeros(mc * 3, np.float32)
        gl = np.zeros(max(lc, 1), np.float32)
        g = _abi.sb_grads(ga.ctypes.data, ge.ctypes.data, gl.ctypes.data)
        self._ck(self._lib.sb_backward(self.field.ctx, C.byref(g)))
        out = dict(albedo=ga.reshape(mc, 3), emissive=ge.reshape(mc, 3), lightScale=gl[:lc].copy())
        if intensities is not None:
            out["intensity"] = out["lightScale"] / np.asarray(intensities, np.float64) * self._lightScale
        return out

    def timings(self) -> dict:
        st = _abi.sb_stats()
        self._ck(self._lib.sb_get_stats(self.field.ctx, C.byref(st)))
        return dict(forwardMs=st.lastForwardRecordMs, backwardMs=st.lastBackwardMs)
