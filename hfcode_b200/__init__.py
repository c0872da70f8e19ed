"""B200-native direct-SCF Fock builder (drop-in for the hfcode fock_build_* path)."""
