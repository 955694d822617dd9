"""Parity oracle: a CPU FP64 restatement of the reference's stream-collide
path (kb_oracle.c).  Test infrastructure only -- never imported by the
product."""
