"""Test infrastructure only: the oracle.

Two CPU implementations of PeriX's PDDO hot path, used only to check results in ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline / reference legs of ``bench.py``:

* ``port``  - ``oracle/_ref/libpddo_oracle.so``, a plain-C restatement (``oracle/pddo_oracle.c``);
* ``ref``   - ``oracle/_ref/libperix_ref.so``, the reference's own hot-path sources compiled by
  ``oracle/Makefile`` together with ``oracle/ref_harness.cpp``.

plus ``oracle/_ref/libperix_ref_cuda.so``: the reference's own CUDA assembly translation unit compiled for
sm_100a (``oracle/ref_cuda_harness.cu``), timed by ``bench.py`` as the GPU reference point and used by the GPU
tests to check the stress-coupled Cahn-Hilliard assembler.

The product (``perix_b200``) never imports this package.
"""
from .lib import (PortOracle, RefMesh, RefEpf, port_available, ref_available, dropin_available,  # noqa: F401
                  bc_program_arrays,
                  ORACLE_DIR, ref_cuda_available, ref_cuda_epf_bench, ref_cuda_stress_ch, ref_cuda_assemble_bench)
