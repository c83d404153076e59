"""B200-native implementation of the ASZ compression hot path."""
