"""B200-native PairHMM forward pass, a drop-in for Biovoltron's PairHMM call."""
