"""CCPi namespace package: the B200-native iterative reconstruction path."""
