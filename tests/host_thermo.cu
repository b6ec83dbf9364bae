// Test infrastructure: a host build of the device thermodynamics (csrc/thermo.cuh) through
// the evaluator the GPU entry point athad_thermo_eval runs on the device (k_thermo.cu,
// eval_one), for tests/test_thermo_host_cpu.py.
#include "../athad_cond_b200/csrc/k_thermo.cu"

extern "C" int host_thermo_arity(int fn) { return athad::arity(fn); }

// fn: an ATHAD_THERMO_* id; in: n tuples of arity(fn) doubles; out: n results.  Returns 0, or
// 1 for an unknown fn.
extern "C" int host_thermo_eval(int fn, int n, const double* in, double* out)
{
    const int a = athad::arity(fn);
    if (a == 0) return 1;
    for (int q = 0; q < n; q++) out[q] = athad::eval_one(fn, in + (long long)q * a);
    return 0;
}
