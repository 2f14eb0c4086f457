// ORACLE — test infrastructure only (see fields.h).
// Linked into oracle/_ref/libstwo_cuda_ref.so beside the reference's own AIR
// kernels (evaluate_wide_fibonacci.cu, evaluate_poseidon_constraint.cu). Those
// read a write-or-accumulate flag that the reference's component dispatcher
// defines; the dispatcher is not built here, so the flag is defined here, set
// to accumulate as the dispatcher sets it for proving (constraint-framework/
// src/prover/component_prover.rs:466: should_accumulate = true).
bool g_should_accumulate_host = true;
