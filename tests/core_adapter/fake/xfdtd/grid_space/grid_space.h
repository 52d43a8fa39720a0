#pragma once
#include "xfdtd/fake_core.h"
