"""Drop-in stencil classes with the reference's names and call signatures."""
