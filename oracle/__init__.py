"""CPU oracle for the Fock build -- test infrastructure only (see oracle.cpp)."""
