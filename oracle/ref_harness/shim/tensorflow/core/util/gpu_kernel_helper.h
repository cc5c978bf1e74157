// Empty stand-in for a TensorFlow header (test infrastructure).
#pragma once
