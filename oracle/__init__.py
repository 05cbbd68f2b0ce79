"""CPU oracle for IFDM_Code's leap-frog Schroedinger-Poisson path.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, by ``__graft_entry__.smoke()``
as the checker, and by ``bench.py``'s cpu_baseline / reference legs.  The product
package ``ifdm_code_b200`` never imports it.

* ``liboracle.so`` (``ifdm_oracle.c``): C restatement of the reference path,
  FP64, with its own FFT (``fft64.c``) and quadrature (``qags.c``).
* ``_ref/BECMPI_ref``: the reference's own unmodified sources compiled against
  single-rank MPI / FFTW / GSL shims (``shim/``), built by ``Makefile`` from the
  reference tree when it is present.
"""

from .pyoracle import IC_EXACT, IC_REF1, Oracle, OracleArgs, build, oracle_constants, ref_binary  # noqa: F401
