"""CPU oracle for hydroflux solver-2d (test infrastructure only; see hf_oracle.hpp)."""
