"""B200-native batched AFQMC walker step (the hot path of bkesk/SAFIRE) behind a C ABI.

    safire_b200.build   - nvcc recipe of the sm_100a library (_lib/libsafire_afqmc.so)
    safire_b200.capi    - ctypes binding of include/afqmc_c.h
    safire_b200.afqmc   - Python mirror of the reference operator API over the C ABI
    safire_b200.driver  - run_afqmc-style step loop (orthogonalisation, comb, measurement)
    safire_b200.synth   - seeded synthetic Hamiltonians / trials of the benchmark workloads
"""
__all__ = ["build", "capi", "afqmc", "driver", "synth"]
