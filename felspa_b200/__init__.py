"""felspa_b200 — B200-native level-set hot path of FELSPA (DG advection +
Hamilton-Jacobi reinitialization) behind a C ABI (include/flsp_dg.h)."""
from . import abi, fields  # noqa: F401
