"""ragdoll_b200: B200-native macroblock analysis / reconstruction for ragdoll's H.264 encoder."""
