"""emagddm_b200: B200-native TET4 Nedelec curl-curl solve path.

Edge numbering and tree-cotree gauge run as host C++; assembly, SpMV and the
Krylov solvers run as hand-written sm_100a CUDA kernels.  Everything is
reached through the C ABI of libemagddm_b200.so (include/emagddm_b200.h);
`emagddm_b200.api` mirrors the reference's classes on top of it.
"""
