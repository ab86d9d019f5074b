"""CPU oracle of the DoNOF.jl RI hot path -- test infrastructure only.

``native`` wraps the C/OpenMP restatement (liboracle.so built from
donof_oracle.c by the Makefile here); ``gnof`` and ``orbital`` are numpy
restatements of the functional, occupation and optimiser layers.  Only the
test suite, the smoke check and the benchmark's CPU-baseline leg use it.
"""
