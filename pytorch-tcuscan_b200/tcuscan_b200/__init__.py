"""B200-specific additions on top of the reference interface: the autotuner,
persistent batched launches and the serving loop."""
