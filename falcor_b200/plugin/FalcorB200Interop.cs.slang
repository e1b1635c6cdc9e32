// FalcorB200Interop.cs.slang -- copies one render-pass channel between its
// Falcor texture and the CUDA-shared staging buffer of the FalcorB200 passes:
// gWords 32-bit words per pixel, rows of gWidth pixels, float or integer view
// (gIsUint).  Bound by FalcorB200Passes.cpp.  (Written for Falcor's Slang
// toolchain; not compiled in this repository, which has no Slang compiler.)
cbuffer CB
{
    uint gWidth;
    uint gHeight;
    uint gWords;
    uint gIsUint;
};

Texture2D<float4> gInTex;
Texture2D<uint4> gInTexU;
RWTexture2D<float4> gOutTex;
RWTexture2D<uint4> gOutTexU;
RWByteAddressBuffer gBuf;

[numthreads(16, 16, 1)]
void texToBuf(uint3 id: SV_DispatchThreadID)
{
    if (id.x >= gWidth || id.y >= gHeight)
        return;
    const uint4 v = gIsUint != 0 ? gInTexU[id.xy] : asuint(gInTex[id.xy]);
    const uint base = (id.y * gWidth + id.x) * gWords * 4;
    for (uint k = 0; k < gWords; k++)
        gBuf.Store(base + 4 * k, v[k]);
}

[numthreads(16, 16, 1)]
void bufToTex(uint3 id: SV_DispatchThreadID)
{
    if (id.x >= gWidth || id.y >= gHeight)
        return;
    const uint base = (id.y * gWidth + id.x) * gWords * 4;
    uint4 v = uint4(0, 0, 0, 0);
    for (uint k = 0; k < gWords; k++)
        v[k] = gBuf.Load(base + 4 * k);
    if (gIsUint != 0)
        gOutTexU[id.xy] = v;
    else
        gOutTex[id.xy] = asfloat(v);
}
