"""B200-native per-batch spike-sorting hot path (Kilosort4 template matching)."""
