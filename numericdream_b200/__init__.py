"""NumericDream B200: the distance-estimator sphere-tracing pass as sm_100a CUDA."""
