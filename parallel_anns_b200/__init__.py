"""B200-native best-first search over NSG proximity graphs (PANNS search path)."""
