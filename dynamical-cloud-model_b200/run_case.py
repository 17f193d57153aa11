"""Run K time steps of a named seeded case through the C-ABI and print the
solver iterations and device time of each step.  A small driver for
profiling single kernels (ncu -k ... on a few steps) and for quick checks.

    python dynamical-cloud-model_b200/run_case.py --case warm_bubble \
        --precision 1 --steps 1 [--host-loop] [--viscous] [--profile]

Cases: warm_bubble (256x256x128), sheared_convection (512x512x256, 8 tracers),
kelvin_helmholtz (128x1x64), or warm_bubble_IPxJPxKP /
sheared_convection_IPxJPxKP for other sizes.  --host-loop drives the
pressure solve from the host (the same kernels; a profiler sees every
launch, which it cannot inside the graph-driven solve's conditional loop);
--graphs 2 keeps the graphs but launches without programmatic dependent
launch.
--output FILE writes the reference's netCDF output before every
--output-every steps and reports the host time of each write call.
--precond 1 gives the mixed form Chebyshev-weighted sweeps on
[--precond-lo, 2].  --viscous switches the Smagorinsky subgrid model on in
sources (cvis 0.23,
z0 = z0th = 0.1 m); --profile prints the device time per kernel class over
the steps after the first.
"""
import argparse
import importlib.util
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))


def load():
    if "dcm_b200" in sys.modules:
        return sys.modules["dcm_b200"]
    spec = importlib.util.spec_from_file_location(
        "dcm_b200", os.path.join(HERE, "__init__.py"), submodule_search_locations=[HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dcm_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def make_case(cases, name):
    if name == "warm_bubble":
        return cases.warm_bubble()
    if name == "sheared_convection":
        return cases.sheared_convection()
    if name == "kelvin_helmholtz":
        return cases.kelvin_helmholtz()
    for stem, fn in (("warm_bubble_", cases.warm_bubble),
                     ("sheared_convection_", cases.sheared_convection)):
        if name.startswith(stem):
            ip, jp, kp = (int(x) for x in name[len(stem):].split("x"))
            return fn(ip=ip, jp=jp, kp=kp)
    raise SystemExit("unknown case " + name)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="warm_bubble")
    ap.add_argument("--precision", type=int, default=1, choices=[0, 1])
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--host-loop", action="store_true")
    ap.add_argument("--graphs", type=int, default=1, choices=[0, 1, 2],
                    help="solver loops: 1 graph-driven, 2 graph-driven without programmatic "
                         "dependent launch, 0 host-polled (as --host-loop)")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--viscous", action="store_true")
    ap.add_argument("--precond", type=int, default=0, choices=[0, 1])
    ap.add_argument("--precond-lo", type=float, default=0.05)
    ap.add_argument("--inner-tol", type=float, default=0.1,
                    help="mixed form: the reliable-update factor")
    ap.add_argument("--fuse", type=int, default=None, choices=[0, 1],
                    help="FP32 preconditioner: separate sweeps (0) or the fused kernel (1)")
    ap.add_argument("--profile", action="store_true")
    ap.add_argument("--output", default=None,
                    help="netCDF file written before every --output-every steps")
    ap.add_argument("--output-every", type=int, default=1)
    args = ap.parse_args()
    dcm = load()
    from dcm_b200 import cases
    c = make_case(cases, args.case)
    core = dcm.DynamicalCore(c.grid, device=args.device)
    if args.host_loop or args.graphs != 1:
        core.solver_graphs(0 if args.host_loop else args.graphs)
    if args.fuse is not None:
        core.set_launch_shape(1, fuse=args.fuse)
    kw = dict(nq=c.nq, c_s=c.c_s, c_e=c.c_e) if c.nq else {}
    if args.viscous:
        kw["viscous"] = dict(lamsq=cases.mixing_length_sq(c.grid, 0.23, 0.1), z0=0.1, z0th=0.1)
    core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                      precision=args.precision, precond=args.precond,
                      precond_lo=args.precond_lo, inner_tol=args.inner_tol, **kw)
    core.driver_start()
    out = dcm.Output(core, args.output) if args.output else None
    t_write = []
    for s in range(args.steps):
        if args.profile and s == min(1, args.steps - 1):
            core.profile(True)  # after the first step (module loading, first-call set-up)
        if out and s % args.output_every == 0:
            t0 = time.perf_counter()
            out.write(s * c.dt)
            t_write.append((time.perf_counter() - t0) * 1e3)
        st = core.step(1)
        print("%s precision %d step %d: %d iterations (%d updates, %d restarts), "
              "err %.3e, %.2f ms" % (c.name, args.precision, s + 1, st.iters_last,
                                     st.updates_last, st.restarts_last, st.err_last,
                                     st.ms_total), flush=True)
    if out:
        t0 = time.perf_counter()
        out.close()
        print("output: %d records, host ms per write call %s, close (drain) %.1f ms" % (
            len(t_write), " ".join("%.2f" % t for t in t_write),
            (time.perf_counter() - t0) * 1e3), flush=True)
    if args.profile:
        for name, (ms, n) in core.profile_read().items():
            if n:
                print("  %-9s %9.3f ms  %6d launches" % (name, ms, n))
    core.close()


if __name__ == "__main__":
    main()
