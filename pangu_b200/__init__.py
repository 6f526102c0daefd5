"""B200-native GRMHD stage engine (PANGU's per-RK-stage hot path)."""
