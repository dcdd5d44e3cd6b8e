#pragma once
#include "../glm_stub.hpp"
