"""B200-native (sm_100a) se_e2_a energy/force/virial path of DeePMD-kit.

Kernels live in ``lib/libdpb200.so`` (sources in ``csrc/``, C-ABI in
``include/dpb200.h``); this package is the host-side mirror of the reference's
operator interface. Importing it loads the library and registers
``torch.ops.deepmd.tabulate_fusion_se_a`` (+ grad ops); it fails loudly if the
library has not been built. The directory name is not a Python identifier, so
the package is imported under the name ``deepmd_kit_lr_pt_b200`` (see
``__graft_entry__.load_package``).
"""

from . import _capi, ops  # noqa: F401

_capi.lib()
ops.register_torch_ops()

__all__ = ["ops"]
