// kpp_b200 CUDA target of the KPP generator: util/util has no device part (the
// kernel does its vector operations and computes SUN itself and passes it to
// Update_RCONST).
