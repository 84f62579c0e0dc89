"""B200-native (sm_100a) matrix-free IMEX-DG operators for the Atmospheric_Flows dynamical core."""
