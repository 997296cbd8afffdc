"""B200-native CUDA backend for the torchls block-sparse LM/GN inner loop."""
