"""B200-native implementation of HiReNSI's explicit 3D elastic FWI time loop."""
