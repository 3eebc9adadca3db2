"""Test infrastructure: the CPU stand-ins for the device kernels live in
oracle/host_kernels.py (built on the oracle); this module re-exports them
for the `host_only` fixture and the host-backend API tests."""
from oracle.host_kernels import fft_items, install, mog_items  # noqa: F401
