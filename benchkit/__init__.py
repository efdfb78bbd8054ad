"""Benchmark and test support for the geraf_b200 RF operators; not part of the
library.

* ``scenes``      seeded synthetic radar scenes (virtual arrays, point scatterers,
                  IF synthesis) standing in for the reference's unreleased data;
* ``sdf``         random-initialised NeuS SDF network and the tracer inputs it gives;
* ``stage1``      a GeRaF stage-1 RF training step on those synthetic inputs;
* ``stage1_eval`` the equal-error comparison of its arithmetic forms;
* ``probes``      FP32 peak probes (the roofline denominators) and the sincosf
                  identity check, in their own library ``libgeraf_probe.so``.
"""
import os
import sys

_PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "geraf-sens_b200")
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)
