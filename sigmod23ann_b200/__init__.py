"""B200 k-NN graph builder with the method of the SIGMOD'23 contest solution
parkertimmins/sigmod23ann: recursive 2-means bucketing, all-pairs inside
buckets into bounded neighbour sets, neighbour-of-neighbour refinement -- all
as sm_100a CUDA kernels behind the C ABI in include/knng.h."""
from .api import (  # noqa: F401
    EXPORTED,
    JobInfo,
    KnngContext,
    KnngError,
    KnngServer,
    Params,
    Stats,
    construct_result,
    default_params,
    job_reservation,
    kd_params,
    load_library,
)
