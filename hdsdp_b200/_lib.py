"""ctypes binding of libhdsdp_b200.so (the in-tree CUDA build).

The library has no CPU path: loading fails loudly when the shared object is
missing, and HDSDPCreate refuses to create a solver without a CUDA device.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhdsdp_b200.so")

# Every entry point declared in include/hdsdp.h, include/hdsdp_user_data.h and
# include/hdsdp_b200.h.
EXPORTS = [
    "HDSDPCreate", "HDSDPInit", "HDSDPSetCone", "HDSDPSetDualObjective", "HDSDPOptimize",
    "HDSDPSetIntParam", "HDSDPSetDblParam", "HDSDPGetRowDual", "HDSDPGetConeValues",
    "HDSDPCheckSolution", "HDSDPClear", "HDSDPDestroy",
    "HUserDataCreate", "HUserDataSetConeData", "HUserDataChooseCone", "HUserDataClear",
    "HUserDataDestroy",
    "HDSDPGetStatus", "HDSDPGetIterCount", "HDSDPSetPrimalRefinement", "HDSDPSetPrecision",
    "HDSDPSetSparseSlack", "HDSDPGetSparseSlackInfo", "HDSDPSetSparseSchur", "HDSDPGetSparseSchurInfo", "HDSDPSetSchurLDL", "hdsdpb_ldl_solve",
    "hdsdpb_sparse_analyse",
    "hdsdpb_sparse_cholesky", "hdsdpb_sparse_congruence",
    "HDSDPGetIterLog", "HDSDPGetTimers", "HDSDPAdjoint",
    "hdsdpb_schur_probe", "hdsdpb_ratio_probe", "hdsdpb_cholesky", "hdsdpb_cholesky_batch", "hdsdpb_cholesky_noalloc", "hdsdpb_cholesky_inverse_factor", "hdsdpb_inverse", "hdsdpb_gemm",
    "hdsdpb_kernel_timing", "hdsdpb_gridsync_probe", "hdsdpb_launch_count", "hdsdpb_alloc_calls", "hdsdpb_release_cached_memory",
    "hdsdpb_kstat_enable", "hdsdpb_kstat_read", "hdsdpb_split_gemm", "hdsdpb_cholesky_solve", "HReadSDPA",
    # the conic callback interface and the KKT manager (include/hdsdp_conic.h)
    "HConeCreate", "HConeGetVarBufferDim", "HConeSetData", "HConeProcData", "HConePresolveData", "HConeClear",
    "HConeDestroy", "HConeView", "HConeDetectFeature", "HConeSetStart", "HConeUpdate", "HConeRatioTest",
    "HConeGetSymNnz", "HConeAddSymNz", "HConeGetSymMapping", "HConeGetDim", "HConeGetCoeffNorm", "HConeGetObjNorm",
    "HConeBuildSchurComplement", "HConeBuildSchurComplementFixed", "HConeGetLogBarrier",
    "HConeAddStepToBufferAndCheck", "HConeCheckIsInterior", "HConeCheckIsInteriorExpert", "HConeReduceResi",
    "HConeSetPerturb", "HConeGetPrimal", "HConeGetDual", "HConeComputeATimesX", "HConeComputeTraceCX",
    "HConeScalByConstant",
    "HKKTCreate", "HKKTInit", "HKKTBuildUp", "HKKTBuildUpExtraCone", "HKKTBuildUpFixed", "HKKTExport",
    "HKKTFactorize", "HKKTSolve", "HKKTRegularize", "HKKTClear", "HKKTDestroy", "HKKTGetMatrix",
]

_lib = None


def load():
    """Load the CUDA library, raising if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libhdsdp_b200.so is missing: run __graft_entry__.build() "
                           "(this library has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp, ip, dp, i, d = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int, C.c_double
    sig = {
        "HDSDPCreate": ([C.POINTER(vp)], i),
        "HDSDPInit": ([vp, i, i], i),
        "HDSDPSetCone": ([vp, i, vp], i),
        "HDSDPSetDualObjective": ([vp, dp], None),
        "HDSDPOptimize": ([vp, i], i),
        "HDSDPSetIntParam": ([vp, i, i], None),
        "HDSDPSetDblParam": ([vp, i, d], None),
        "HDSDPGetRowDual": ([vp, dp, dp, dp], i),
        "HDSDPGetConeValues": ([vp, i, dp, dp, dp], None),
        "HDSDPCheckSolution": ([vp, dp], i),
        "HDSDPClear": ([vp], None),
        "HDSDPDestroy": ([C.POINTER(vp)], None),
        "HUserDataCreate": ([C.POINTER(vp)], i),
        "HUserDataSetConeData": ([vp, i, i, i, ip, ip, dp], None),
        "HUserDataChooseCone": ([vp], i),
        "HUserDataClear": ([vp], None),
        "HUserDataDestroy": ([C.POINTER(vp)], None),
        "HDSDPGetStatus": ([vp], i),
        "HDSDPGetIterCount": ([vp], i),
        "HDSDPSetPrimalRefinement": ([vp, i], None),
        "HDSDPSetPrecision": ([vp, i], None),
        "HDSDPSetSparseSlack": ([vp, i], None),
        "HDSDPGetSparseSlackInfo": ([vp, dp], None),
        "HDSDPSetSparseSchur": ([vp, i], None),
        "HDSDPGetSparseSchurInfo": ([vp, dp], None),
        "HDSDPSetSchurLDL": ([vp, i], None),
        "hdsdpb_ldl_solve": ([i, dp, dp, dp, ip], i),
        "hdsdpb_sparse_analyse": ([i, i, ip, ip, i, dp, ip], i),
        "hdsdpb_sparse_cholesky": ([i, i, ip, ip, dp, i, i, dp], i),
        "hdsdpb_sparse_congruence": ([i, i, ip, ip, dp, dp, dp, dp, dp], i),
        "HDSDPGetIterLog": ([vp, i, dp, dp, dp, dp, dp, ip], i),
        "HDSDPGetTimers": ([vp, dp], None),
        "HDSDPAdjoint": ([vp, dp, dp, dp, dp, dp], i),
        "hdsdpb_schur_probe": ([i, i, ip, ip, dp, dp, d, i, dp, dp, dp, dp], i),
        "hdsdpb_ratio_probe": ([i, i, ip, ip, dp, dp, d, dp, d, dp, dp], i),
        "hdsdpb_cholesky": ([i, dp, dp, dp], i),
        "hdsdpb_cholesky_batch": ([i, i, i, dp, dp, dp, dp, ip], i),
        "hdsdpb_cholesky_noalloc": ([i, dp, dp, dp], i),
        "hdsdpb_inverse": ([i, dp, dp], i),
        "hdsdpb_cholesky_inverse_factor": ([i, dp, dp, dp], i),
        "hdsdpb_cholesky_solve": ([i, dp, dp, dp], i),
        "HReadSDPA": ([C.c_char_p] + [vp] * 13, i),
        "hdsdpb_gemm": ([i, i, i, d, dp, i, i, dp, i, i, d, dp, i], i),
        "hdsdpb_kernel_timing": ([i, i, i, dp], i),
        "hdsdpb_gridsync_probe": ([i, i, dp], i),
        "hdsdpb_launch_count": ([], C.c_longlong),
        "hdsdpb_alloc_calls": ([], C.c_longlong),
        "hdsdpb_release_cached_memory": ([], None),
        "hdsdpb_kstat_enable": ([i], i),
        "hdsdpb_split_gemm": ([i, i, i, dp, i, i, dp, i, i, dp, i], i),
        "hdsdpb_kstat_read": ([i, C.POINTER(C.c_longlong), dp, dp], i),
        "HConeCreate": ([C.POINTER(vp)], i),
        "HConeGetVarBufferDim": ([vp], i),
        "HConeSetData": ([vp, vp], i),
        "HConeProcData": ([vp], i),
        "HConePresolveData": ([vp], i),
        "HConeClear": ([vp], None),
        "HConeDestroy": ([C.POINTER(vp)], None),
        "HConeView": ([vp], None),
        "HConeDetectFeature": ([vp, dp, ip, dp], None),
        "HConeSetStart": ([vp, d], None),
        "HConeUpdate": ([vp, d, dp], None),
        "HConeRatioTest": ([vp, d, dp, d, i, dp], i),
        "HConeGetSymNnz": ([vp], C.c_int64),
        "HConeAddSymNz": ([vp, i, ip], None),
        "HConeGetSymMapping": ([vp, i, ip], None),
        "HConeGetDim": ([vp], i),
        "HConeGetCoeffNorm": ([vp, i], d),
        "HConeGetObjNorm": ([vp, i], d),
        "HConeBuildSchurComplement": ([vp, vp, i], i),
        "HConeBuildSchurComplementFixed": ([vp, vp, i, i], i),
        "HConeGetLogBarrier": ([vp, d, dp, i, dp], i),
        "HConeAddStepToBufferAndCheck": ([vp, d, i, ip], i),
        "HConeCheckIsInterior": ([vp, d, dp, ip], i),
        "HConeCheckIsInteriorExpert": ([vp, d, d, dp, d, i, ip], i),
        "HConeReduceResi": ([vp, d], None),
        "HConeSetPerturb": ([vp, d], None),
        "HConeGetPrimal": ([vp, d, dp, dp, dp, dp], None),
        "HConeGetDual": ([vp, dp, dp], None),
        "HConeComputeATimesX": ([vp, dp, dp], None),
        "HConeComputeTraceCX": ([vp, dp], d),
        "HConeScalByConstant": ([vp, d], None),
        "HKKTCreate": ([C.POINTER(vp)], i),
        "HKKTInit": ([vp, i, i, C.POINTER(vp)], i),
        "HKKTBuildUp": ([vp, i], i),
        "HKKTBuildUpExtraCone": ([vp, vp, i], i),
        "HKKTBuildUpFixed": ([vp, i, i], i),
        "HKKTExport": ([vp, dp, dp, dp, dp, dp, dp, dp], None),
        "HKKTFactorize": ([vp], i),
        "HKKTSolve": ([vp, dp, dp], i),
        "HKKTRegularize": ([vp, d], None),
        "HKKTClear": ([vp], None),
        "HKKTDestroy": ([C.POINTER(vp)], None),
        "HKKTGetMatrix": ([vp, dp], i),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L
