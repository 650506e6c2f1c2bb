"""oxideav_h266_b200 — B200-native H.266/VVC in-loop filter chain.

Host-side mirror of the oxideav-h266 crate's filter API (src/deblock.rs,
src/sao.rs, src/alf.rs, src/lmcs.rs, src/ctu.rs:11822) over the C ABI in
include/oxideav_h266_b200.h.  The compute path is the CUDA library built from
csrc/ for sm_100a; nothing here falls back to CPU arithmetic.
"""
from . import abi, workloads  # noqa: F401
