"""tfhe_b200: B200-native TFHE gate bootstrapping behind the tfhe v1.1 gate API.

The product is the C-ABI library tfhe_b200/libtfhe_b200.so (include/tfhe_b200.h, include/tfhe.h);
this package is its Python mirror (tfhe_b200.api)."""
from . import api  # noqa: F401
from .api import (FP64, SPLIT_FP32, CloudKey, NetlistMulti, SecretKey, default_params,  # noqa: F401
                  fft_slot_order, gate_batch_multi, kernel_launches, keygen, large_params, load_ciphertexts, load_cloud_keyset, load_params,
                  load_secret_keyset, make_params, save_ciphertexts, save_cloud_keyset, save_params,
                  save_secret_keyset)
