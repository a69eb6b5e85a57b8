#include "mlp.cuh"
