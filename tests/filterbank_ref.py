"""The FP64 restatement of the batched FIR -> cascaded-biquad filter bank and its
adjoint lives in the oracle package (oracle/filterbank64.py); re-exported here for
the tests that import it by this name."""
from oracle.filterbank64 import (bank_adjoint, bank_forward, channel_adjoint, channel_forward,  # noqa: F401
                                 stable_sections)
