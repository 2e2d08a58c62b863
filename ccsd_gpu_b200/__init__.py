"""B200-native CCSD analytic-gradient hot path.

Drop-in entry points with the signatures of the ``ccsd_gpu`` prototype:
``compute_int2e_gpu``, ``compute_int2e_ip1_gpu`` (``ccsd_gpu_b200.cuda``),
``solve_lambda_gpu``, ``grad_elec_gpu`` and ``compute_ml_ccsd_forces_gpu``.
All numerical work runs in ``libccsdb200.so`` (sm_100a) through a C ABI.
"""
from .cuda.int2e_gpu import compute_int2e_gpu  # noqa: F401
from .cuda.int2e_ip1_gpu import compute_int2e_ip1_gpu  # noqa: F401
from .cuda.basis import _check_mol  # noqa: F401
