// FalcorB200MeshData.cs.slang -- per-vertex shading normals and tangents of
// one mesh, read from the scene's vertex data as Scene/MeshIO.cs.slang reads
// positions (MeshIO.cs.slang:53-59); Scene::getMeshVerticesAndIndices gives
// the rest.  Bound by FalcorB200Passes.cpp (makeDescFromScene).  (Written for
// Falcor's Slang toolchain; not compiled in this repository.)
import Scene.Scene;

struct MeshAttribLoader
{
    uint vertexCount;
    uint vbOffset;
    RWStructuredBuffer<float3> normals;
    RWStructuredBuffer<float4> tangents;
};

ParameterBlock<MeshAttribLoader> gLoader;

[numthreads(256, 1, 1)]
void main(uint3 id: SV_DispatchThreadID)
{
    if (id.x >= gLoader.vertexCount)
        return;
    const StaticVertexData v = gScene.getVertex(id.x + gLoader.vbOffset);
    gLoader.normals[id.x] = v.normal;
    gLoader.tangents[id.x] = v.tangent;
}
