"""chainamps_b200: the ChainAMPS two-site DMRG hot path on B200 (sm_100a).

The product is the CUDA library ``libchainamps_b200.so`` (C ABI in
``include/chainamps_b200.h``); ``chainamps_b200.capi`` is its host-side
mirror of the reference's call surface.  Importing any API name loads the
library and fails loudly when it is not built -- there is no CPU fallback.
"""
__all__ = ["Context", "TwoVertexComponents", "SVDResult", "Block", "MPXTensor", "MPXIndexSpec", "CmpsError",
           "upload_block", "iDMRG", "fDMRG", "run_excited_fdmrg", "DEFAULT_PROJECTOR_WEIGHT", "CMPS_FP64",
           "CMPS_SPLIT_TF32", "CMPS_SPLIT_BF16", "CMPS_ORDER_AUTO", "CMPS_ORDER_FOLDED", "CMPS_ORDER_CANONICAL", "CMPS_FORM_NONE", "CMPS_FORM_FOLDED_TC",
           "CMPS_FORM_CANONICAL_FP32", "CMPS_FORM_CANONICAL_TC", "version"]


def __getattr__(name):
    if name in __all__:
        from . import capi
        return getattr(capi, name)
    raise AttributeError(name)
