"""Test infrastructure: the CPU FP64 oracle of the RTMC path (see ptrans_oracle.h)."""
