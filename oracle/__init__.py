"""CPU oracle for the FFT-operator contact solve -- TEST INFRASTRUCTURE ONLY.

This package restates, in numpy/scipy, the reference algorithms of ASPHER's
``backend="fft"`` / ``backend="periodic"`` contact solve so that the CUDA
product path can be checked against it.  It is imported only by ``tests/``,
by ``__graft_entry__.smoke()`` (as the checker) and by ``bench.py``'s CPU
baseline / reference arm.  The product (``aspher_b200``) never imports it and
has no CPU fallback.

Why a restatement and not the reference itself: the reference is a C++17
library whose every header includes Eigen (``include/contact_solver.hpp:3``),
and Eigen is not installed here (its CMake would download it,
``CMakeLists.txt:28-40``; there is no network).  A library the path needs
that is absent makes the reference unbuildable in this container, so the
oracle follows the reference sources line by line instead:

* ``love.py``      -- ``src/boussinesq_kernel.cpp:60-106`` (Love cell integral)
* ``operators.py`` -- ``src/fft_operator.cpp:18-138``,
                      ``src/periodic_fft_operator.cpp:11-101``
* ``precond.py``   -- ``src/stencil_precond.cpp:19-109,199-220``,
                      ``src/fourier_precond.cpp:12-116``
* ``solver.py``    -- ``src/contact_solver.cpp:31-60,69-99,150-587``
* ``nested.py``    -- ``src/nested_solve.cpp:27-990`` (fft/periodic,
                      with the active-set levels of ``:72-518``)
* ``api.py``       -- ``python/bindings.cpp:115-234,362-432,637-879``

FFT arithmetic: the reference runs pocketfft (vendored at
``third_party/pocketfft/pocketfft_hdronly.h``, BSD).  The oracle calls
``scipy.fft`` (scipy 1.18), whose backend is the same pocketfft C++ code, so
transforms agree with the reference's to roundoff.

Parity pins (see ``tests/test_oracle_*.py``): the Love fixture of the
reference's ``tests/data/love_reference.txt`` (worst rel err <= 1e-12), the
golden stencil weights of ``tests/test_stencil.cpp:21-33`` (5e-6), the exact
self term of ``tests/test_kernel.cpp:21-24``, dense == FFT matvec
(``tests/test_fft.cpp:20-39``), periodic Fourier modes / Westergaard
(``tests/test_periodic.cpp:16-129``) and the certification gates of
``tests/test_certification*.``.
"""

from . import love, operators, precond, solver, nested, api  # noqa: F401
