"""B200-native SuperCountingBloom insert / query / spectrum path (sm_100a CUDA behind a C ABI)."""
