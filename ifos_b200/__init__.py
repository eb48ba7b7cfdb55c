"""B200-native shot solver for the IFOS2D forward/adjoint propagation path."""
