"""B200-native PDLP engine: a drop-in for the reference solver's PDLP dispatch
target (``pdlp::PdlpSolver::solve``), built from hand-written sm_100a CUDA
kernels behind a C ABI (``include/pdlpgpu.h``)."""
from .lp import CompiledLp, PdlpOptions, PdlpResult, PdlpStatus, SparseMatrix  # noqa: F401
