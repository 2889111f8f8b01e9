"""FibreNet-B200: FibreNet's per-timestep particle dynamics on B200."""
