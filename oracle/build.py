"""ORACLE — test infrastructure only.

Builds the CPU checkers used by tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg:

* oracle/liboracle.so      the CPU restatement (pm_oracle.cpp), always;
* oracle/_ref/libpmref.so  the reference's own kernel sources
                           (cvt/cl/kernel/pmhstereo.cl, PDDiffTensor.cl,
                           PDDROFDiffTensor.cl, PDDHuberDiffTensor.cl,
                           pyr/pyrdown.cl, pyr/pyrupmul.cl, VPMStereo.cl,
                           gradxy.cl, SVPMFlow.cl)
                           rewritten by translate.py and
                           compiled against clshim.h, when the reference tree is
                           present (it is not on GPU machines; the built .so
                           travels with the checkout instead).

The reference checkout is found at $CVT_REFERENCE_ROOT, or given as
`python oracle/build.py --reference DIR`; by default it is a directory named
`reference` beside this repository.

Both are built with -O2 -ffp-contract=off -fno-fast-math: every C operator
rounds once, so results do not depend on the compiler's contraction choices.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_kernels(root=None):
    """cvt/cl/kernel of the reference checkout: `root`, else $CVT_REFERENCE_ROOT, else the
    directory `reference` beside this repository"""
    root = root or os.environ.get("CVT_REFERENCE_ROOT") or os.path.join(os.path.dirname(os.path.dirname(HERE)),
                                                                        "reference")
    return os.path.join(root, "cvt", "cl", "kernel")



CXXFLAGS = ["-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared", "-std=c++17"]


def _run(cmd):
    subprocess.run(cmd, check=True)


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build_oracle(force=False):
    out = os.path.join(HERE, "liboracle.so")
    srcs = [os.path.join(HERE, f) for f in ("pm_oracle.cpp", "pm_oracle.h", "pm_libm.h", "pm_hostloop.h")]
    if force or _stale(out, srcs):
        _run(["g++"] + CXXFLAGS + ["-o", out, srcs[0]])
    return out


def build_ref(force=False, kernel_dir=None):
    kernel_dir = kernel_dir or reference_kernels()
    refdir = os.path.join(HERE, "_ref")
    out = os.path.join(refdir, "libpmref.so")
    if not os.path.isdir(kernel_dir):
        return out if os.path.exists(out) else None
    os.makedirs(refdir, exist_ok=True)
    cls = ["pmhstereo.cl", "PDDiffTensor.cl", "PDDROFDiffTensor.cl", "PDDHuberDiffTensor.cl", "VPMStereo.cl",
           "gradxy.cl", "SVPMFlow.cl"]
    deps = [os.path.join(kernel_dir, f) for f in cls + ["RNG.cl", "MWC64X.cl", "Matrix3.cl"]]
    pyr = ["pyrdown.cl", "pyrupmul.cl"]
    deps += [os.path.join(kernel_dir, "pyr", f) for f in pyr]
    glue = [os.path.join(HERE, f) for f in ("ref_pmh.cpp", "ref_pd.cpp", "ref_pyr.cpp", "ref_vpm.cpp", "ref_svpm.cpp", "ref_driver.cpp")]
    hdrs = [os.path.join(HERE, f) for f in ("clshim.h", "ref_exec.h", "pm_hostloop.h", "pm_libm.h", "translate.py")]
    if not (force or _stale(out, deps + glue + hdrs)):
        return out
    for f in cls:
        _run([sys.executable, os.path.join(HERE, "translate.py"), kernel_dir, f, os.path.join(refdir, f + ".cpp")])
    for f in pyr:
        _run([sys.executable, os.path.join(HERE, "translate.py"), os.path.join(kernel_dir, "pyr"), f,
              os.path.join(refdir, f + ".cpp")])
    _run(["g++"] + CXXFLAGS + ["-w", "-Wno-narrowing", "-I", HERE, "-o", out] + glue)
    return out


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("-f", action="store_true", help="rebuild even when up to date")
    ap.add_argument("--reference", help="root of the reference checkout")
    a = ap.parse_args()
    print(build_oracle(force=a.f))
    print(build_ref(force=a.f, kernel_dir=reference_kernels(a.reference) if a.reference else None))
