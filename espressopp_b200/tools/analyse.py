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
    NPart = system.storage.getNRealParticles()
    print("total time: %.1f" % (end_time - start_time))
    print("number of particles:", NPart)
    print("number of verlet-list pairs:", vl.totalSize())
    print("neighbours per particle: %.2f" % (vl.totalSize() / float(NPart)))
    print("number of verlet-list builds:", vl.builds)
    print("number of resorts:", integrator.getNumResorts())
