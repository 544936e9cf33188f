"""B200-native LBM per-timestep path (placeholder until the CUDA library lands)."""
