"""Host side of the B200 presearch engine: parameters, synthetic workloads
and ctypes bindings of libghostz_b200.so."""
