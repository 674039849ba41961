"""Python access to the B200 OWT-Krylov solve path (ctypes over include/owtk.h).

`native` binds the C ABI of lib/libowtk_b200.so (loaded on first use);
`problems` generates the seeded synthetic systems of the benchmark
configurations; `learned`, `train_learned` and `checkpoint` train, save and
load the learned preconditioner.  Import the submodules explicitly.
"""
