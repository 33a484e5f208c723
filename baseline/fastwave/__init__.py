"""The reference's GPU path (rave-sim fast-wave: its CUDA kernels and cuFFT
plan class, compiled unmodified from the reference checkout) driven over the
engine's workloads, for the GPU baseline of bench.py. ``build`` compiles it
where the reference checkout is present; ``run`` times it in a separate
process."""
