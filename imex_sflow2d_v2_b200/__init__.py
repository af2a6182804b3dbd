"""B200-native IMEX_SfloW2D time step: C ABI (libimexgpu.so) + Python host side."""
