"""B200 engine for the all-pairs alignment -> distance step of DSC-SPIDAL/csharp.

Local Smith-Waterman-Gotoh (Salsa.SmithWatermanMPI / Salsa.SmithWatermanMS) and global
Needleman-Wunsch (Salsa.NeedlemanWunschTPL) with affine gaps, each pair reduced to the
reference's Int16 distance, computed by CUDA kernels for sm_100a behind the C ABI in
``include/swgb200.h``.  This package is the host-side mirror of the reference's aligner and
block-handler interface over that ABI.
"""
from .core import (Block, Engine, NUCLEIC, NW, PROTEIN, PairwiseAlignment, Range, ScoringMatrix,
                   SmithWatermanGotoh, SWG_MPI, SWG_MS, block_is_computed, block_partition,
                   measure_int_peak, pack_sequences, range_partition)
from .core import JUKES_CANTOR, KIMURA2, MIN_MAX_NORM_SCORE, PERCENT_IDENTITY
from .lib import SwError

__all__ = ["Block", "Engine", "NUCLEIC", "NW", "PROTEIN", "PairwiseAlignment", "Range",
           "ScoringMatrix", "SmithWatermanGotoh", "SWG_MPI", "SWG_MS", "block_is_computed",
           "block_partition", "measure_int_peak", "pack_sequences", "range_partition",
           "PERCENT_IDENTITY", "KIMURA2", "JUKES_CANTOR", "MIN_MAX_NORM_SCORE", "SwError"]
