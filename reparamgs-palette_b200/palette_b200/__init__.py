"""Extensions around the drop-in ``gsplatcu`` operators: cameras and synthetic
scenes, autograd functions (the reference's and a fused full-adjoint one),
precision helpers and the palette-edit serving loop."""
