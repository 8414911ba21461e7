"""B200-native EPSR minimum-image pair path.

Device kernels (sm_100a) behind a C ABI (``include/epsr_gpu.h``, ``libepsr_gpu.so``), with
host bindings that keep the reference translation's routine names and signatures:

* ``box`` / ``configs`` -- host arrays and seeded synthetic systems;
* ``device.DeviceBox`` -- device-resident state and the pair-path calls;
* ``transforms`` -- gensq, stog, fit_expansion;
* ``dropin`` -- installs the routines into the reference's modules (epsr26).
"""

__version__ = "0.1.0"
