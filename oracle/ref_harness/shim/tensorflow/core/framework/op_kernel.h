// Stand-in (test infrastructure): see op.h.
#pragma once
#include "tensorflow/core/framework/op.h"
