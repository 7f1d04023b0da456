"""CPU oracle for the iDFT solve: test infrastructure only (see oracle.h)."""
