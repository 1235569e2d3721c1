"""B200-native TRTT forward/back projector pair (placeholder, filled below)."""
