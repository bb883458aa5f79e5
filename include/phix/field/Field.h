#pragma once
#include "field/ScalarField.h"
