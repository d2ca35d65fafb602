"""The reference voxelizer on the GPU for A/B tests: its compiled CUDA
extension (oracle/_ref/, built by oracle/build_ref.py from its sources) with
its autograd glue and a torch restatement of its preprocess and binning
(oracle/ref_cuda.py)."""
from oracle.ref_cuda import REF, RefFn, RefVoxelizer, reference_step  # noqa: F401
