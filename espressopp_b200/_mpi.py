"""``espressopp.MPI.COMM_WORLD`` of the reference's scripts (mpi4py there): the rank and
size of the torch.distributed world when one is initialised (one process per GPU under
torchrun), else a single process.  Scripts use it to size the node grid:
``decomp.nodeGrid(espressopp.MPI.COMM_WORLD.size, box, rc, skin)``."""


class _CommWorld:
    @staticmethod
    def _dist():
        try:
            import torch.distributed as dist
        except ImportError:
            return None
        return dist if dist.is_available() and dist.is_initialized() else None

    @property
    def size(self):
        d = self._dist()
        return d.get_world_size() if d else 1

    @property
    def rank(self):
        d = self._dist()
        return d.get_rank() if d else 0

    def Get_size(self):
        return self.size

    def Get_rank(self):
        return self.rank


class MPI:
    COMM_WORLD = _CommWorld()
