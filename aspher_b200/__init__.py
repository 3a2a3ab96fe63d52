"""aspher_b200: ASPHER's FFT-operator contact solve on NVIDIA B200 (sm_100a).

Public API (drop-in for the reference's fft / periodic backends):
  ContactSolver(grid_size, domain_size=1.0, E_star=1.0, ..., backend="fft"|"periodic")
      .matvec(p), .solve(gap, p_nominal, tol, max_iter, use_pr, precond, p_init)
  solve_nested(grid_size, gap, p_nominal, ..., backend="fft"|"periodic", precision=...)
  ContactResult (pressure, contact_area, iterations, fw_error, penetration_error, status, ...)
Lower level: Operator (device matvec), solve_device (device tensors in / out),
solve_device_batch / solve_device_batch_mixed (many problems, one loop graph).
Derivatives: adjoint(op, pressure, dL/dp), contact_pressure (torch.autograd).
Tangential: TangentialOperator (the Cerruti block on the device).
"""

from ._lib import AspherError, LIB_PATH  # noqa: F401
from .api import (ContactResult, ContactSolver, Operator, solve_device,  # noqa: F401
                  solve_device_batch, solve_device_batch_mixed, solve_device_mixed, stencil_taps)
from .adjoint import adjoint, contact_pressure  # noqa: F401
from .nested import solve_nested  # noqa: F401
from .surfaces import self_affine_gap  # noqa: F401
from .tangential import TangentialOperator  # noqa: F401

__all__ = ["ContactSolver", "ContactResult", "Operator", "solve_device", "solve_device_mixed",
           "solve_device_batch", "solve_device_batch_mixed",
           "solve_nested", "adjoint", "contact_pressure",
           "stencil_taps", "self_affine_gap", "AspherError", "TangentialOperator"]
