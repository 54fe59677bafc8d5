"""CPU FP64 restatement of MLegS's pseudo-spectral transform-and-step path.

TEST INFRASTRUCTURE ONLY.  This package is the parity oracle and the timed
CPU baseline.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it;
the product library (``mlegs_b200``) never does, and has no CPU fallback.

Every function restates one routine of the reference (Fortran 90) and cites
the file:line it follows (paths relative to the MLegS project root).  The
reference itself cannot be compiled in this environment (no Fortran
compiler, MPI, FFTW or MKL), so parity is pinned through the known-answer
checks the reference's own tests and notes state (divxm analytic case,
q-vortex log term = -0.5, PF orthonormality, FFF->PPP->FFF identity, ETD
4x4 vs. matrix exponential) and through 50-digit mpmath tables of the
associated Legendre functions built with the reference's LEG_TBL3
recurrence (tests/golden/).

Layout conventions (0-based, C order, same index meaning as the reference):
  FFF  E[n, m, k]  shape (NRCHOPDIM, NTCHOPDIM, NXCHOPDIM)
  PFF  E[r, m, k]  shape (NDIMR,     NTCHOPDIM, NXCHOPDIM)
  PFP  E[r, j, z]  shape (NDIMR,     NDIMTH,    NX)
  PPP  E[r, j, z]  shape (NDIMR,     NDIMTH,    NX)
Single process: the reference's MPI offsets INR/INTH/INX are all zero.
"""

from .grid import Grid, Field, FFF, PFF, PFP, PPP  # noqa: F401
