"""B200-native AV2 in-loop filter + film-grain path (the post-reconstruction
stage of the rav2d decoder): deblocking, CDEF+CCSO, loop restoration
(NS-Wiener, PC-Wiener, GDF) and film grain as sm_100a CUDA kernels behind a
C ABI (include/rav2d_gpu.h)."""
