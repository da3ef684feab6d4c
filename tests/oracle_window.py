"""A window solver backed by the oracle's periodic stepper, with the
EngineWindow methods (pysweep_b200.distributed): lets the row-slab and
share-split drivers run on CPU in the tests (the oracle is only the checker
of the GPU path; here it stands in for the GPU's window)."""
import numpy as np

import oracle


class OracleWindow:
    """Window solver with the EngineWindow methods, backed by the oracle."""

    def __init__(self, equation, globals_, its):
        self.eq, self.g, self.its = equation, globals_, its
        self.u = self.prev = None

    def set_global(self, name, value):
        pass

    def set_window(self, field):
        f = np.array(field, dtype=np.float64)
        if f.ndim == 4:  # oldest level first, as Engine.set_state takes them
            self.prev, self.u = f[0].copy(), f[-1].copy()
        else:
            self.u, self.prev = f.copy(), f.copy()

    def run(self, nlevels, gts0):
        _, self.u, self.prev = oracle.standard(self.eq, self.u, self.g, self.its, nlevels,
                                               gts0=gts0, frames=False, prev=self.prev)

    def _level(self, level):
        return self.u if level == 0 else self.prev

    def get_rows(self, row0, nrows, level):
        return self._level(level)[:, row0:row0 + nrows].copy()

    def set_rows(self, row0, rows, level):
        self._level(level)[:, row0:row0 + rows.shape[1]] = rows

    def synchronize(self):
        pass

    def close(self):
        pass
