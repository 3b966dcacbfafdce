"""B200-native FMM cell-interaction kernels for Octo-Tiger."""
