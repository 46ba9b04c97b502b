"""B200-native lane sweeps of ESPice's GPU lane path (see include/espice_lanes.h)."""
