// Driver for the reference's compositing known-answer routine testRender()
// (SVRF/VolumeFieldRender.cu:111-183), which prints its results with printArray.
// Test infrastructure only: the printed values become tests/golden/kat_test_render.json.
void testRender();

int main()
{
    testRender();
    return 0;
}
