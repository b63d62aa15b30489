"""tools.timers.show (src/tools/timers.py:53)."""


def show(alltimers, precision=1):
    names = ["run", "pair", "FENE", "angle", "comm1", "comm2", "int1", "int2", "resort", "other"]
    t = alltimers[0]
    fmt = "%%s = %%.%df" % precision
    for n, v in zip(names, t):
        print(fmt % (n, v))
