// Project-written stand-in for the reference's voxelizer/voxelizer.h, whose util.h needs
// trimesh2 and glm (absent here).  The solver sources that include it use none of its
// declarations; the standard headers it pulls in are kept.
#pragma once
#include <array>
#include <iostream>
#include <utility>
#include <vector>
