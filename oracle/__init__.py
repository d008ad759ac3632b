"""FP64 CPU oracle of the channel-DNS hot path - test infrastructure only."""
