"""The reference's E1 linear-case gates (engine/oracle/src/criteria.rs:7-41), its iteration-growth gate between
mesh sizes (e3_summarize.rs:28-35) and its effective-bandwidth figure (compare.rs:9-11, 63-68), restated as test
checkers for the GPU's block-Jacobi PCG on the E1 systems (tests/test_gpu_e1.py)."""

FORCING_LIMIT = 1e-2             # a converged f32 solve cuts the true f64 residual at least 100x
F32_ITERATION_RATIO_LIMIT = 1.5  # f32 CG may take at most 1.5x the f64 iterations
ITERATION_GROWTH_LIMIT = 3.0     # iterations per mesh halving
SPEEDUP_LIMIT = 10.0             # over one CPU core running f64 PCG
EMULATION_ITERATION_SLACK = 0.05
BYTES_PER_BLOCK, BYTES_PER_ROW = 40.0, 196.0


def verdict(status, iterations, true_relative_residual, f64_iterations, emulated_iterations, difference_vs_cpu_f32,
            relative_error, deterministic, cpu_f64_seconds, gpu_solve_ms):
    """criteria.rs:26-41: the per-case flags."""
    same_iterations = abs(iterations - emulated_iterations) <= 2.0 + EMULATION_ITERATION_SLACK * emulated_iterations
    return {
        "converged": status == "converged",
        "forcing_term_ok": true_relative_residual <= FORCING_LIMIT,
        "f32_iterations_ok": iterations <= F32_ITERATION_RATIO_LIMIT * f64_iterations,
        "faithful_to_cpu_f32_emulation": bool(same_iterations and difference_vs_cpu_f32 <= max(2.0 * relative_error, 1e-6)),
        "deterministic": bool(deterministic),
        "speedup_ok": 1e3 * cpu_f64_seconds / gpu_solve_ms >= SPEEDUP_LIMIT,
    }


def growth(iterations_by_size):
    """e3_summarize.rs:28-35 on [(unknowns, iterations), ...]: the ratio between consecutive mesh sizes (smallest
    first) and whether it stays below the limit."""
    rows = sorted(iterations_by_size)
    return [(b[1] / a[1], b[1] / a[1] < ITERATION_GROWTH_LIMIT) for a, b in zip(rows, rows[1:])]


def effective_bandwidth_gbs(blocks, rows, iterations, gpu_ms):
    """compare.rs:63-68: compulsory traffic of one PCG iteration (40 B per block, 196 B per row) over the time."""
    return (BYTES_PER_BLOCK * blocks + BYTES_PER_ROW * rows) * iterations / (gpu_ms * 1e6)
