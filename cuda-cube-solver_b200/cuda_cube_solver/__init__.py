"""B200-native optimal solver for the 3x3 Rubik's cube (half-turn metric).

Drop-in for the reference's ``cuda_cube_solver`` package: same modules (``cubie``, ``geometry``,
``coords``, ``kinds``, ``facelets``, ``table``, ``solver``, CLI), with the GPU work done by
``libccs``, a C-ABI library of hand-written CUDA kernels for sm_100a (see ``native``).
"""
