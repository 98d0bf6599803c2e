"""B200-native explicit RHS + SSP-RK3 step of a 3D compressible Navier-Stokes solver."""
