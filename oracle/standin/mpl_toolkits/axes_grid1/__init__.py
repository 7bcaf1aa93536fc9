"""TEST INFRASTRUCTURE ONLY: inert stand-in."""
