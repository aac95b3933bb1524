"""Cases the reference program is built for (oracle/build_ref.py) and run on
(tests/golden/make_golden.py, bench.py's reference arm).  TEST INFRASTRUCTURE.

Every case uses T_hot = 1, T_cold = 0, gravity 1 and beta = 0.01/LY (free-fall
velocity 0.1).  continue_step > 0 makes the reference start from restart files
(src/initial.cu:110-205), which is how seeded states are fed to it.
"""
NEVER = 1_000_000_000

REF_CASES = {
    # parity cases on small non-cubic closed boxes
    "w12_rest50": dict(lx=12, ly=10, lz=8, continue_step=0, nend=50, ndiag=10, nnuout=10,
                       rayleigh=1.0e5, prandtl=0.71),
    "w12_s1": dict(lx=12, ly=10, lz=8, continue_step=100, nend=101, rayleigh=1.0e5, prandtl=0.71),
    "w12_s2": dict(lx=12, ly=10, lz=8, continue_step=100, nend=102, rayleigh=1.0e5, prandtl=0.71),
    "w12_s1000": dict(lx=12, ly=10, lz=8, continue_step=100, nend=1100, ndiag=100, nnuout=100,
                      rayleigh=1.0e5, prandtl=0.71),
    "w24_s1000": dict(lx=24, ly=16, lz=20, continue_step=100, nend=1100, ndiag=100, nnuout=100,
                      rayleigh=1.0e5, prandtl=0.71),
    # long run at the 64^3 benchmark grid (Ra 1e5): 10,000 steps from a seeded state
    "c0_s10000": dict(lx=64, ly=64, lz=64, continue_step=100, nend=10100, nnuout=1000,
                      rayleigh=1.0e5, prandtl=0.71),
    # timing cases: the seeded conduction state of conduction_restart (seed
    # 1000, noise 1e-3; bench.py's engine workload) fed through the restart
    # path, 3 and 203 steps, at 256^3 Ra 1e7 and 64^3 Ra 1e5
    "c1_r3": dict(lx=256, ly=256, lz=256, continue_step=100, nend=103, rayleigh=1.0e7, prandtl=0.71),
    "c1_r203": dict(lx=256, ly=256, lz=256, continue_step=100, nend=303, rayleigh=1.0e7, prandtl=0.71),
    "c0_r3": dict(lx=64, ly=64, lz=64, continue_step=100, nend=103, rayleigh=1.0e5, prandtl=0.71),
    "c0_r203": dict(lx=64, ly=64, lz=64, continue_step=100, nend=303, rayleigh=1.0e5, prandtl=0.71),
}

# timing binaries of one grid: (grid tag, short run, long run); the per-step
# time is the difference of their printed GPU times over 200 steps
TIMING_SETS = {
    "c1": ("c1_r3", "c1_r203"),
    "c0": ("c0_r3", "c0_r203"),
}
TIMING_SEED = 1000
