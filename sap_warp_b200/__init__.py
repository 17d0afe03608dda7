"""B200-native SAP contact step (drop-in for the SAP step of mardigiorgio/sap_warp).

The solve runs only through the native library libsapb.so (hand-written
sm_100a CUDA behind the C ABI of include/sapb.h); torch supplies device memory
and streams.
"""

__all__ = ["scenes"]
