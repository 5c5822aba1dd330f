"""B200-native Cahn-Hilliard step loop for phasefield5d (sm_100a CUDA behind a C ABI)."""
__version__ = "0.1.0"
