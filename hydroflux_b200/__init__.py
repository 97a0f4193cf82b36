"""hydroflux_b200: B200-native (sm_100a, FP64) explicit step of hydroflux solver-2d."""
