"""Drop-in classes with the reference's module layout (models/block.py, models/bold_model_pytorch.py)."""
