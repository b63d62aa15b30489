"""tools.analyse.info / final_info (src/tools/analyse.py:24-76)."""
import sys


def info(system, integrator, per_atom=False):
    from .. import analysis
    NPart = analysis.NPart(system).compute()
    T = analysis.Temperature(system).compute()
    P = analysis.Pressure(system).compute()
    Pij = analysis.PressureTensor(system).compute()
    step = integrator.step
    Ek = (3.0 / 2.0) * NPart * T
    Etotal = 0.0
    if per_atom:
        tot = "%5d %10.4f %10.6f %10.6f %12.8f" % (step, T, P, Pij[3], Ek / NPart)
    else:
        tot = "%5d %10.4f %10.6f %10.6f %12.3f" % (step, T, P, Pij[3], Ek)
    tt = ""
    for k in range(system.getNumberOfInteractions()):
        e = system.getInteraction(k).computeEnergy()
        Etotal += e
        tot += (" %12.8f" % (e / NPart)) if per_atom else (" %12.3f" % e)
        tt += ("     e%i/N    " % k) if per_atom else ("      e%i     " % k)
    tot += (" %12.8f" % (Etotal / NPart + Ek / NPart)) if per_atom else (" %12.3f" % (Etotal + Ek))
    tt += "   etotal/N  " if per_atom else "    etotal   "
    tot += " %12.8f\n" % system.bc.boxL[0]
    tt += "    boxL     \n"
    if step == 0:
        head = " step      T          P        Pxy         ekin/N  " if per_atom else \
            " step      T          P        Pxy          ekin   "
        sys.stdout.write(head + tt)
    sys.stdout.write(tot)


def final_info(system, integrator, vl, start_time, end_time):
    """Final report (src/tools/analyse.py:66-76): the integrator's timers, the Verlet
    list's size, neighbours per particle and builds, the step count, and the wall time
    of the one process that drives the GPU (the reference prints its MPI rank count and
    the time per rank on that line)."""
    from .. import analysis
    from . import timers
    NPart = analysis.NPart(system).compute()
    timers.show(integrator.getTimers(), precision=3)
    sys.stdout.write("Total # of neighbors = %d\n" % vl.totalSize())
    sys.stdout.write("Ave neighs/atom = %.1f\n" % (vl.totalSize() / float(NPart)))
    sys.stdout.write("Neighbor list builds = %d\n" % vl.builds)
    sys.stdout.write("Integration steps = %d\n" % integrator.step)
    sys.stdout.write("CPUs = %i CPU time per CPU = %.5f\n" % (1, end_time - start_time))
