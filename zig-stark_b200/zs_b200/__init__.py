"""zs_b200: a B200 (sm_100a) backend for zig-stark's M31 DEEP-FRI commitment path."""
from . import wire, workload  # noqa: F401
