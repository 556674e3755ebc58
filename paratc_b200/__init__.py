"""B200-native ParaTC hot path: CUDA kernels for sm_100a behind a C ABI
(include/paratc.h), with a thin Python mirror of the reference's channel
interface in paratc_b200.lib.  Importing the package loads nothing; the CUDA
library is loaded by paratc_b200.lib.load()."""
__all__ = ["abi", "cases", "lib"]
