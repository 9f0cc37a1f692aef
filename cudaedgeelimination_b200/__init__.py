"""B200-native edge-elimination screen: JV candidates, exact k-opt leaf cost matrices and the
HT c,d root screen as sm_100a kernels behind a C ABI (include/cee.h, libcee.so)."""
from .snapshot import CEIL_2D, EUC_2D, GraphSnapshot  # noqa: F401
from .api import (  # noqa: F401
    CD_TASK_DTYPE, KOPT_TASK_DTYPE, Candidate, Context, BuildKOptReconnectTable, ClearJvCudaCache,
    ClearKOptCostCudaCache, CudaBackendAvailable, EvaluateKOptTemplateCostsCuda, FindJvCandidatesCuda,
    HtCdCudaAvailable, KOptCostCudaAvailable, KOptReconnectTable, ScreenHtCdCandidatesCuda, device_count,
    ClearHtReplyCudaCache, EvaluateHtEndRepliesCuda, EvaluateHtHamiltonRepliesCuda, HtEndReplyCudaAvailable,
    HtHamiltonReplyCudaAvailable,
    JV_EPOCH_METRICS_DTYPE, JV_PROOF_RECORD_DTYPE, TuningCache, content_hash, jv_proof, write_active_edges,
    write_jv_proof,
)
