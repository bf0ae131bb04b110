"""Package path of the reference rasterizer (``cuda_kernel_rasterize``), so
``from cuda_kernel_rasterize.cuda_rasterizer import ...`` in renderer.py:5
resolves to the sm_100a implementation."""
