"""B200-native SuperCountingBloom insert / query / spectrum path.

The compute path is libscb_b200.so: hand-written CUDA kernels for sm_100a behind the C ABI of
include/scb.h.  This package is the host-side mirror of the reference crate's public API
(super-counting-bloom 0.1.0) over that ABI, plus seeded workload generators.
"""
from .api import (  # noqa: F401
    AddReport,
    BuildIndexReport,
    ChannelClosed,
    CounterBits,
    FastxOpen,
    FilterOnlySpectrumEstimate,
    InternalState,
    InvalidConfig,
    InvalidIndexFormat,
    Io,
    QueryFastaReport,
    SequenceAbundanceSummary,
    StreamEstimateReport,
    StreamEstimateStats,
    SuperCountingBloomBuilder,
    SuperCountingBloomConfig,
    SuperCountingBloomError,
    SuperCountingBloomIndex,
    SuperCountingBloomReport,
    SuperCountingBloomServer,
    SuperCountingBloomStats,
    WorkerPanic,
    estimate_spectrum_from_fastx,
    estimate_spectrum_from_fastx_pair,
    for_each_fastx_record,
    pack_sequences,
    set_strategy,
    stream_estimates_from_fastx,
    stream_estimates_from_fastx_pair,
    write_spectrum,
)
from .filter import (  # noqa: F401
    FrozenSuperCountingBloom,
    PackedSeqVec,
    SuperCountingBloom,
    canonical_kmer,
    xorshift_u64,
)
