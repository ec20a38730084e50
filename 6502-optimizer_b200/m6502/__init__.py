"""m6502 -- host-side mirror of the 6502 superoptimizer's API over the B200
engine (libm6502gpu.so).

  inst    -- pkg/inst: opcodes, Disassemble, ByteSize, Cycles, parse_assembly
  engine  -- pkg/search/verifier.go: QuickCheck, MidCheck, ExhaustiveCheck(+Masked),
             FlagDiff, Fingerprint, ShouldPrune; the Engine context and batch calls
  search  -- pkg/search/search.go: Config, Run, SearchSingle(Masked)
  result  -- pkg/result: Rule, DeadFlagDesc, JSON and JSONL output
"""
from . import _lib, inst, mlp, result  # noqa: F401
from ._lib import (CHECK_ALL, CHECK_EXH, CHECK_MID, CHECK_QC, COST_HAMMING, COST_REF,  # noqa: F401
                   EXH_BRUTE, EXH_CONES, SEM_CUDA, SEM_GO, SWEEP_FULL, SWEEP_REFERENCE, M6502Error)
from .engine import (DeadAll, DeadNone, Engine, ExhaustiveCheck, ExhaustiveCheckMasked,  # noqa: F401
                     FlagDiff, Fingerprint, MidCheck, MidCheckMasked, QuickCheck,
                     QuickCheckMasked, ShouldPrune, default_engine)
from .search import Config, Run, SearchSingle, SearchSingleMasked  # noqa: F401
