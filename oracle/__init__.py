"""Test infrastructure: the CPU oracle of the hot path (see oracle.h). Not product code."""
