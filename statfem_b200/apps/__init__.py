"""Front ends that run the reference applications' input files unchanged."""
