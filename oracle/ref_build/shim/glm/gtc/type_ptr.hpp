// glm/gtc/type_ptr.hpp of the project-written glm subset (test infrastructure only, oracle/_ref):
// make_vec2 / make_vec3 / make_mat4 live in ../glm.hpp.
#pragma once
#include "../glm.hpp"
