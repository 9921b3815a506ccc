"""speedball_b200 — B200-native DDGI probe update (sm_100a CUDA behind a C ABI).

Public entry points mirror the reference facade: ``installSpeedballGI`` and
``createProbeField`` (speedball_b200.field); scenes are described with
``speedball_b200.scene`` and packed into the reference's pooled layouts.
"""
from .field import ProbeField, SpeedballGIHandle, createProbeField, installSpeedballGI  # noqa: F401

__all__ = ["ProbeField", "SpeedballGIHandle", "createProbeField", "installSpeedballGI"]
