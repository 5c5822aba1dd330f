"""Drop-in mirror of phasefield5d.solver's step-loop surface, backed by the CUDA library."""
