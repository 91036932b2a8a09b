/* CenterlineExtraction3D.h -- correctly spelled alias of CenterlineExctraction.h. */
#pragma once
#include "CenterlineExctraction.h"
