// Host set-up of the kernels' parameter block (see setup.cpp).
#pragma once
#include <string>
#include "../../include/mb3d_cu.h"
#include "devparams.h"

namespace mb3dcu {
// 0: the backend renders the scene; 1: it cannot (why); < 0: a bad scene.
int unsupported_reason(const mb3d_cu_scene &sc, std::string &why);
// CalcParams::new for the card: 0 or a negative status (err says why).
int setup_params(const mb3d_cu_scene &sc, DevParams &p, std::string &err);
}  // namespace mb3dcu
