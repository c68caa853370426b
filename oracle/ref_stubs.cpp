// Link stub for the reference CPU build in oracle/_ref (test infrastructure only).
//
// Scene::addTriangleMesh (src/Scene.cpp:55-75) calls TriangleMesh::getTriangle, whose
// definition lives in src/triangleMesh.cpp next to the assimp importer; libassimp is not
// available, so the harness never loads meshes and this stub satisfies the linker.
#include "triangleMesh.h"

Triangle* TriangleMesh::getTriangle(int) { return nullptr; }
