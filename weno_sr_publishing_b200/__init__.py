"""B200-native WENO5-SR / WENO5-JS finite-volume solver (drop-in for the reference's 2D Euler path)."""
