"""openjij_b200 — B200-native single-spin-flip annealing (SA / SQA) behind
OpenJij's sampler API."""
