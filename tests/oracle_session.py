"""The oracle behind the step-consumer interface a GpuSession offers
(jacobian_async / normal_equations / lm_step / lsq_step / eval_population),
so the host-side solver logic runs on CPU against FP64 restatements."""
import numpy as np

from oracle import api as O


class OracleStepSession(O.Oracle):
    def jacobian_async(self, w_e=1.0, w_s=0.0):
        F = self.eval(w_e, w_s, want=("F",))["F"]
        try:
            J = self.jacobian_analytic(w_e, w_s)
        except Exception:
            J = self.jacobian_fd(w_e, w_s)
        self._JtJ, self._Jtr = O.normal_equations(J, F)
        self._obj = float(F @ F)

    def normal_equations(self):
        return self._JtJ.copy(), self._Jtr.copy(), self._obj

    def lm_step(self, lam, mode=0):
        return O.lm_step(self._JtJ, self._Jtr, lam, mode)

    def lsq_step(self, ridge=0.0):
        return O.lsq_step(self._JtJ, self._Jtr, ridge)
