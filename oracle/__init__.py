"""CPU oracle for the particle-mesh (PM) step of DiscoDJNative `run_nbody`.

TEST INFRASTRUCTURE ONLY. This package is a plain restatement of the
reference's algorithm (numpy float64, plus the small C helper `cpm.c` for sizes
numpy cannot reach in seconds). It exists to check the CUDA library: only the
tests, `__graft_entry__.smoke()` and the CPU-baseline leg of `bench.py` may
import it, and never as the thing measured or shipped. The product path
(`discodj.jl_b200`) must not import anything from here.

Parity of this oracle is pinned against the reference's own golden vectors,
`native/DiscoDJNative/test/reference/jax_nbody_reference.h5` (JAX DISCO-DJ,
float64), converted to `tests/golden/jax_nbody_reference.npz`, at the
reference's tolerances (`native/DiscoDJNative/test/nbody_parity_tests.jl:17-61`):
timetables < 1e-13, stepper coefficients < 1e-12, PM acceleration < 1e-12 and
full runs < 1e-11 relative (max-abs / max-abs).

Modules
-------
cosmology  Cosmology, compute_timetables, growth ODE, timetable lookups
           (`src/cosmology/Cosmology.jl`, `src/cosmology/growth.jl`,
           `src/nbody/timetables.jl`)
nbody      stepper_coefficients, run_nbody, nbody_ics_lpt, bullfrog_ics
           (`src/nbody/run_nbody.jl`)
pm         PMConfig, PM force with every option (`src/nbody/pm.jl`)
power      evaluate_power_spectrum (`src/analysis/power_spectrum.jl`)
lpt        2LPT/3LPT displacement shapes from an IC potential
           (`src/lpt/nlpt_core.jl`), EH transfer + IC map
           (`src/cosmology/transfer.jl`, `src/ics/grf.jl`)
cpm        ctypes binding of cpm.c (OpenMP scatter / FD gather, float32 and
           float64) used for the larger parity cases and the CPU baseline

All paths above are relative to `native/DiscoDJNative/` in the reference.
"""
