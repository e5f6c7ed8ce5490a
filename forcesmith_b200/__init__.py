"""B200-native objective-evaluation path of Forcesmith (host-side mirror).

The product is the CUDA library behind include/forcesmith_gpu.h; this
package holds its ctypes binding (`gpu`), the shared ABI structs (`abi`)
and the seeded synthetic workloads (`synth`).
"""
from .abi import Dataset, Model, Table, FsError  # noqa: F401
