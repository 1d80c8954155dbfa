"""snuqs_b200: a B200-native state-vector engine behind SnuQS's plugin surface.

* ``snuqs_b200._C`` -- the reference's pybind11 module surface
  (``braket.snuqs._C``: operation, operation.gate_operations, functionals,
  result_types, stream, event, core, core.cuda, DeviceType).
* ``snuqs_b200.capi`` -- ctypes binding of the C ABI (include/snuqs_b200.h).
* ``snuqs_b200.adjoint`` -- adjoint gradients behind ``torch.autograd``.
* ``snuqs_b200.circuits`` -- seeded workload generators.
* ``snuqs_b200.sharding`` -- batches split across ranks (torch.distributed).

The native libraries are built in-tree by ``python -m snuqs_b200.build``.
Without them every engine entry point raises (``import snuqs_b200._C`` fails,
``capi.lib()`` raises ImportError): the engine has no CPU fallback.  The
package itself imports without them so that the build module can run.
"""
from __future__ import annotations

import os

_HERE = os.path.dirname(os.path.abspath(__file__))

__version__ = "0.1.0"
LIB_PATH = os.path.join(_HERE, "libsnuqs_b200.so")
