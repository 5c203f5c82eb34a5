"""rover_b200 -- B200-native quantized graph search behind Rover's C-ABI."""
