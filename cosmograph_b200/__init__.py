"""B200-native BSSN (+dust / +scalar) RK4 evolution for periodic boxes."""
