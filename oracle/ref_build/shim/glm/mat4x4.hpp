// glm/mat4x4.hpp of the project-written glm subset (test infrastructure only, oracle/_ref).
#pragma once
#include "glm.hpp"
