"""B200-native TreePM short-range particle-particle (P2P) force pass.

Host-side mirror of the reference's gpu_entry interface over the C ABI of
libphotons_p2p.so (include/photons_p2p.h). Submodules:
  abi        ctypes declarations of the C ABI
  p2p        Session: the pass on device-resident particles, leaves and lists
  lists      caller-side tree build / walk (libphotons_lists.so)
  workloads  seeded synthetic particle sets and pass configurations
"""
