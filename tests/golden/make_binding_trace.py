"""Record the calls the reference's own ClawSolver2D makes to its step module,
for the binding test (tests/test_gpu_binding.py), into
tests/golden/binding_trace.npz.

The reference's ClawSolver2D.step_hyperbolic (src/pyclaw/classic/solver.py:
498-549) calls ``self.fmod.step2`` / ``step2ds`` with f2py's positional
arguments and passes the Riemann solver as ``self.rp.rpn2._cpointer``.  With
``solver.fmod = pyclaw_b200.classic2`` and Riemann modules whose ``_cpointer``
is a pyclaw_b200 solver, the UNMODIFIED reference host layer (setup,
_apply_bcs, the dt loop, Controller.run) drives the CUDA step: that is the
whole binding.  The reference cannot be imported on the GPU machine, so this
script runs it here -- its examples advection_2d (unsplit, trans_cor: the
``classic_unsplit_trans_cor`` golden) and euler_2d quadrants (split Roe: the
``quadrants_roe`` golden) -- with a recording step module that computes with
the CPU oracle, checks that the run reproduces the reference's golden, and
saves the recorded calls: every call's dt and Courant number, and the full
arguments and results of the first calls (and, for advection, of the last
one).  The GPU test
replays those calls through pyclaw_b200.classic2.

Usage (where the reference tree is mounted; TEST INFRASTRUCTURE only):
    python tests/golden/make_binding_trace.py <path to the reference tree>
    (or set CLAW_REFERENCE)
"""
import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "binding_trace.npz")


def install_reference(ref):
    """The reference's Python host layer as ``clawpack.pyclaw``, with this
    package's Riemann solver objects standing in for ``clawpack.riemann``'s
    modules (names, static tables, constants, rpn2/rpt2._cpointer) and an
    empty ``clawpack.visclaw`` (plotting only)."""
    sys.path.insert(0, ROOT)
    from pyclaw_b200 import riemann as rb

    cp = types.ModuleType("clawpack")
    cp.__path__ = []
    sys.modules["clawpack"] = cp

    rmod = types.ModuleType("clawpack.riemann")
    rmod.__path__ = []
    rmod.static = rb.static
    for s in rb._ALL:
        setattr(rmod, s.name, s)  # the solver objects stand where f2py modules would
        consts = getattr(rb, s.name + "_constants", None)
        if consts is not None:
            cm = types.ModuleType("clawpack.riemann.%s_constants" % s.name)
            cm.__dict__.update(vars(consts))
            setattr(rmod, s.name + "_constants", cm)
            sys.modules[cm.__name__] = cm
    sys.modules["clawpack.riemann"] = rmod
    cp.riemann = rmod

    vis = types.ModuleType("clawpack.visclaw")
    vis.__path__ = []
    vis.colormaps = types.ModuleType("clawpack.visclaw.colormaps")
    sys.modules["clawpack.visclaw"] = vis
    sys.modules["clawpack.visclaw.colormaps"] = vis.colormaps
    cp.visclaw = vis

    src = os.path.join(ref, "src", "pyclaw")
    spec = importlib.util.spec_from_file_location("clawpack.pyclaw", os.path.join(src, "__init__.py"),
                                                  submodule_search_locations=[src])
    pyclaw = importlib.util.module_from_spec(spec)
    sys.modules["clawpack.pyclaw"] = pyclaw
    cp.pyclaw = pyclaw
    spec.loader.exec_module(pyclaw)
    # setup() reloads the f2py module to flush its COMMON blocks
    # (classic/solver.py:229-232); the recorder has none to flush
    sys.modules["clawpack.pyclaw.classic.solver"].reload = lambda m: m
    return pyclaw


class Recorder(types.ModuleType):
    """A step module with f2py's signature (classic/solver.py:527-541) that
    computes with the oracle and records every call."""

    def __init__(self, keep_first):
        super().__init__("binding_recorder")
        self.cparam = types.SimpleNamespace()
        self.calls = []
        self.keep_first = keep_first

    def _record(self, name, args, qold, qin, qout, cfl, rp, ids=0):
        maxm, num_ghost, mx, my, _, _, auxbc, dx, dy, dt, method, mthlim = args[:12]
        rec = {"name": name, "rp": rp.name, "ids": ids, "maxm": maxm, "num_ghost": num_ghost, "mx": mx, "my": my,
               "dx": dx, "dy": dy, "dt": dt, "method": np.array(method), "mthlim": np.array(mthlim),
               "cparam": dict(vars(self.cparam)), "cfl": cfl}
        if len(self.calls) < self.keep_first:
            rec.update(qold=qold.copy(order="F"), qin=qin.copy(order="F"), qout=qout.copy(order="F"))
        self.calls.append(rec)
        self.last = (rec, qold.copy(order="F"), qin.copy(order="F"), qout.copy(order="F"))

    def _cp(self, rp):
        return rp.cparam(vars(self.cparam))

    def step2(self, maxm, num_ghost, mx, my, qold, qbc, auxbc, dx, dy, dt, method, mthlim, aux1, aux2, aux3,
              work, fwave, rpn2, rpt2):
        from oracle import pyoracle
        qin = np.asfortranarray(qbc).copy(order="F")
        qout = qin.copy(order="F")
        cfl = pyoracle.step2(np.asfortranarray(qold), qout, dx, dy, dt, method, mthlim, rpn2.rp_id, self._cp(rpn2),
                             bool(fwave))
        self._record("step2", (maxm, num_ghost, mx, my, qold, qbc, auxbc, dx, dy, dt, method, mthlim),
                     np.asfortranarray(qold), qin, qout, cfl, rpn2)
        return qout, cfl

    def step2ds(self, maxm, num_ghost, mx, my, qold, qbc, auxbc, dx, dy, dt, method, mthlim, aux1, aux2, aux3,
                work, ids, fwave, rpn2, rpt2):
        from oracle import pyoracle
        qin = np.asfortranarray(qbc).copy(order="F")
        qout = qin.copy(order="F")
        cfl = pyoracle.step2ds(np.asfortranarray(qold), qout, dx, dy, dt, method, mthlim, ids, rpn2.rp_id,
                               self._cp(rpn2), bool(fwave))
        self._record("step2ds", (maxm, num_ghost, mx, my, qold, qbc, auxbc, dx, dy, dt, method, mthlim),
                     np.asfortranarray(qold), qin, qout, cfl, rpn2, ids=ids)
        return qout, cfl


def run_case(ref, key, module_path, setup_kw, golden_key, comp, keep_first, keep_last=True):
    spec = importlib.util.spec_from_file_location("ref_example_" + key, module_path)
    ex = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ex)
    claw = ex.setup(**setup_kw)
    claw.output_format = None
    rec = Recorder(keep_first)
    claw.solver.fmod = rec  # the binding: the reference's own solver, this step module
    claw.run()
    q = claw.frames[claw.num_output_times].state.get_q_global()
    gold = np.load(os.path.join(os.path.dirname(module_path), "expected_sols.npy"), allow_pickle=True).item()
    dx, dy = claw.solution.domain.grid.delta
    l1 = dx * dy * np.sum(np.abs(q[comp].reshape([-1]) - gold[golden_key]))
    assert l1 < 1e-6, (key, l1)
    out = {}
    calls = rec.calls
    out[key + "_n"] = np.array(len(calls))
    out[key + "_dt"] = np.array([c["dt"] for c in calls])
    out[key + "_cfl"] = np.array([c["cfl"] for c in calls])
    out[key + "_ids"] = np.array([c["ids"] for c in calls])
    out[key + "_l1_oracle_vs_golden"] = np.array(l1)
    last, qold, qin, qout = rec.last
    keep = [(i, c) for i, c in enumerate(calls[:keep_first])]
    if keep_last:
        keep.append((len(calls) - 1, dict(last, qold=qold, qin=qin, qout=qout)))
    for j, (i, c) in enumerate(keep):
        p = "%s_call%d_" % (key, j)
        out[p + "index"] = np.array(i)
        out[p + "name"] = np.array(c["name"])
        out[p + "rp"] = np.array(c["rp"])
        for f in ("ids", "maxm", "num_ghost", "mx", "my", "dx", "dy", "dt", "cfl"):
            out[p + f] = np.array(c[f])
        out[p + "method"], out[p + "mthlim"] = c["method"], c["mthlim"]
        out[p + "cparam_keys"] = np.array(sorted(c["cparam"]))
        out[p + "cparam_vals"] = np.array([float(c["cparam"][k]) for k in sorted(c["cparam"])])
        # the reference passes qbc with the same contents as qold (classic/solver.py:514,527-541)
        assert np.array_equal(c["qin"], c["qold"])
        out[p + "qold"], out[p + "qout"] = c["qold"], c["qout"]
    out[key + "_kept"] = np.array(len(keep))
    print(key, "calls", len(calls), "oracle L1 vs golden %.3e" % l1)
    return out


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CLAW_REFERENCE")
    if not ref:
        sys.exit("usage: make_binding_trace.py <path to the reference tree> (or set CLAW_REFERENCE)")
    install_reference(ref)
    ex = os.path.join(ref, "examples")
    out = {}
    out.update(run_case(ref, "advection", os.path.join(ex, "advection_2d", "advection_2d.py"),
                        dict(outdir=None, solver_type="classic", dimensional_split=False, transverse_waves=2),
                        "classic_unsplit_trans_cor", 0, keep_first=2))
    out.update(run_case(ref, "quadrants", os.path.join(ex, "euler_2d", "quadrants.py"),
                        dict(riemann_solver="roe"), "quadrants_roe", 0, keep_first=2, keep_last=False))
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
