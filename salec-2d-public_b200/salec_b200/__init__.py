"""B200 (sm_100a) per-timestep mesh update of the SALEc2d impact hydrocode.

The product is the C ABI of ``include/salec_gpu.h`` implemented by the in-tree library
``libsalec_b200.so`` (hand-written CUDA kernels, FP64). This package holds the host-side
mirror used by Python callers and tests:

- ``capi``   ctypes binding of the C ABI (``Simulation`` = one device-resident mesh);
- ``decks``  writer of SALEc2d ``.inp`` decks and EOS key files for seeded synthetic impacts;
- ``fields`` field name lists (state, step inputs, output set);
- ``build``  the nvcc recipe that produces the library.

There is no CPU fallback: loading ``capi`` raises when the library is missing and cannot be built.
"""
