"""g1sim_b200 -- B200-native batched Unitree G1 step (sm_100a CUDA behind a C-ABI)."""
